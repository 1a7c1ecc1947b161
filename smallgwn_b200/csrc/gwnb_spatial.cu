// Spatial queries on the BVH4: unsigned point-to-mesh distance and ray first hit.
//
// smallgwn: the batch entry points include/gwn/gwn_query.cuh:114-282, the traversals
// detail/gwn_query_distance_impl.cuh:40-160 and detail/gwn_query_ray_impl.cuh:376-560, the
// geometric kernels detail/gwn_query_geometry_impl.cuh:49-114 and detail/gwn_query_ray_impl.cuh:
// 63-238. Same traversal order as smallgwn's canonical traversal -- a node's valid children are
// compacted in slot order, sorted near-first by the five-comparator network, leaf children are
// evaluated inside their node, internal children queued far to near with the nearest entered
// directly -- and smallgwn's formulas in its operation order, every sum, quotient and square root
// rounded on its own and dot products, cross products, 2 x 2 determinants and slab bounds fused in
// one fixed pattern of multiply-adds (explicit _rn intrinsics); the oracle restates the same pattern
// with C's fmaf, so results equal it bit for bit (smallgwn leaves contraction to its compiler).
//
// Differences: queries may be taken in Hilbert order of the query points / ray origins (the batch
// writes results at their input positions); node children are read as 128-bit loads and triangles
// from the padded 48-byte records; the stack lives in shared memory; among hits at the same ray
// parameter the lower original primitive id wins (smallgwn keeps whichever its traversal meets
// first); a stack overflow writes NaN (distance) or the overflow status (ray) and sets the BVH's
// device error bit instead of trapping.
#include "gwnb_internal.cuh"

#include <cstring>

#include <cfloat>

namespace gwnb {

int query_order(aabb const *root_bounds, float const *qx, float const *qy, float const *qz, std::uint64_t n,
                std::uint32_t *order, cudaStream_t s, unsigned int *status);

namespace {

// Ray hit record, layout of gwn::gwn_ray_first_hit_result<float, uint32_t> (32 B).
struct ray_hit {
    float t, u, v, nx, ny, nz;
    std::uint32_t primitive_id;
    std::uint32_t status_word; // status in the low byte, zero padding above it
};
static_assert(sizeof(ray_hit) == 32);
static_assert(sizeof(ray_hit) == sizeof(gwnb_ray_hit_f32));

struct spatial_params {
    float4 const *nodes; // node_count x 8 float4 (the 128-byte smallgwn node)
    std::uint64_t node_count;
    triangle48 const *tri48;
    std::uint32_t const *primitive_indices;
    std::uint64_t primitive_count;
    std::uint64_t root_ref;
    float const *qx, *qy, *qz; // query points or ray origins
    float const *dx, *dy, *dz; // ray directions
    std::uint32_t const *order; // sorted position -> query index (nullptr: identity)
    float *distance;
    ray_hit *hits;
    std::uint32_t *stat_nodes, *stat_tris;
    std::uint64_t n;
    float culling_band;
    float t_min, t_max;
    int stack_cap; // entries of this thread's stack column (the BVH's internal stack bound, at least 1)
    unsigned int *status;
    unsigned long long *next_item; // persistent kernels: first unclaimed sorted position (zeroed per launch)
};

// ---- arithmetic: every product, sum and quotient rounded on its own, fused multiply-adds in one
// fixed pattern (the oracle evaluates the same pattern with C's fmaf) -----------------------------

struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 operator+(v3 a, v3 b) {
    return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ v3 operator-(v3 a, v3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
// a * s + c per component
__device__ __forceinline__ v3 fma3(v3 a, float s, v3 c) {
    return {__fmaf_rn(a.x, s, c.x), __fmaf_rn(a.y, s, c.y), __fmaf_rn(a.z, s, c.z)};
}
// detail/gwn_query_vec3_impl.cuh:109-121, fused: x x' first, then y and z accumulated
__device__ __forceinline__ float dot(v3 a, v3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
// a b - c d with the second product rounded first
__device__ __forceinline__ float dop(float a, float b, float c, float d) { return __fmaf_rn(a, b, -__fmul_rn(c, d)); }
__device__ __forceinline__ v3 cross(v3 a, v3 b) { return {dop(a.y, b.z, a.z, b.y), dop(a.z, b.x, a.x, b.z), dop(a.x, b.y, a.y, b.x)}; }

// Vertices of a padded record, reconstructed as v0 + e (detail/gwn_query_distance_impl.cuh:20-33).
__device__ __forceinline__ void record_vertices(triangle48 const *t48, std::uint64_t i, v3 &a, v3 &b, v3 &c) {
    float4 const A = __ldg(&t48[i].a);
    float4 const B = __ldg(&t48[i].b);
    float4 const C = __ldg(&t48[i].c);
    a = {A.x, A.y, A.z};
    b = a + v3{A.w, B.x, B.y};
    c = a + v3{B.z, B.w, C.x};
}

// Packed reference of child slot s of a node (the second 128-bit half of the 32-byte child).
__device__ __forceinline__ std::uint64_t child_ref(float4 const *nd, int s) {
    float4 const B = __ldg(nd + 2 * s + 1);
    return (static_cast<std::uint64_t>(__float_as_uint(B.w)) << 32) | __float_as_uint(B.z);
}

// Candidate payload: internal child -> its node index; leaf child -> k_leaf_payload | slot (the
// leaf's range is re-read from the node when it is visited).
constexpr std::uint32_t k_leaf_payload = 0x80000000u;

// Fixed-size candidate list: the node's surviving children compacted in slot order, then sorted by
// key (static register indexing throughout).
struct cand4 {
    float key[4];
    std::uint32_t pay[4];
    __device__ __forceinline__ void put(int k, float d, std::uint32_t v) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j == k) {
                key[j] = d;
                pay[j] = v;
            }
    }
    __device__ __forceinline__ void cswap(int l, int r) {
        if (key[l] > key[r]) {
            float const tk = key[l];
            key[l] = key[r];
            key[r] = tk;
            std::uint32_t const tp = pay[l];
            pay[l] = pay[r];
            pay[r] = tp;
        }
    }
    // detail/gwn_query_distance_impl.cuh:105-119: sentinels, then the five-comparator network.
    __device__ __forceinline__ void sort(int count) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j >= count) {
                key[j] = __int_as_float(0x7f800000);
                pay[j] = k_invalid_u32;
            }
        cswap(0, 1);
        cswap(2, 3);
        cswap(0, 2);
        cswap(1, 3);
        cswap(1, 2);
    }
};

// Payload of a surviving child, or k_invalid_u32 for an internal child outside the node array
// (skipped, as smallgwn skips it when popped).
__device__ __forceinline__ std::uint32_t child_payload(std::uint64_t ref, int s, std::uint64_t node_count) {
    if (ref_leaf(ref))
        return k_leaf_payload | static_cast<std::uint32_t>(s);
    return ref_offset(ref) < node_count ? static_cast<std::uint32_t>(ref_offset(ref)) : k_invalid_u32;
}

// ---- unsigned distance ------------------------------------------------------------------------

// std::max(v, 0) keeping smallgwn's NaN behaviour (the first operand is returned when unordered).
__device__ __forceinline__ float pos(float v) { return (v < 0.0f) ? 0.0f : v; }

// detail/gwn_query_geometry_impl.cuh:104-114
__device__ __forceinline__ float aabb_d2(v3 q, float4 A, float4 B) {
    float const dx = __fadd_rn(pos(__fsub_rn(A.x, q.x)), pos(__fsub_rn(q.x, A.w)));
    float const dy = __fadd_rn(pos(__fsub_rn(A.y, q.y)), pos(__fsub_rn(q.y, B.x)));
    float const dz = __fadd_rn(pos(__fsub_rn(A.z, q.z)), pos(__fsub_rn(q.z, B.y)));
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// Squared point-triangle distance by the Voronoi-region tests of Ericson, "Real-Time Collision
// Detection" (2005) 5.1.5, in the operation order of detail/gwn_query_geometry_impl.cuh:49-100.
__device__ __forceinline__ float point_triangle_d2(v3 p, v3 a, v3 b, v3 c) {
    v3 const ab = b - a, ac = c - a, ap = p - a;
    float const d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f)
        return dot(ap, ap);
    v3 const bp = p - b;
    float const d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3)
        return dot(bp, bp);
    float const vc = dop(d1, d4, d3, d2);
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float const v = __fdiv_rn(d1, __fsub_rn(d1, d3));
        v3 const q = p - fma3(ab, v, a);
        return dot(q, q);
    }
    v3 const cp = p - c;
    float const d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6)
        return dot(cp, cp);
    float const vb = dop(d5, d2, d1, d6);
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float const w = __fdiv_rn(d2, __fsub_rn(d2, d6));
        v3 const q = p - fma3(ac, w, a);
        return dot(q, q);
    }
    float const va = dop(d3, d6, d5, d4);
    float const d43 = __fsub_rn(d4, d3), d56 = __fsub_rn(d5, d6);
    if (va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f) {
        float const w = __fdiv_rn(d43, __fadd_rn(d43, d56));
        v3 const q = p - fma3(c - b, w, b);
        return dot(q, q);
    }
    float const denom = __fdiv_rn(1.0f, __fadd_rn(__fadd_rn(va, vb), vc));
    float const v = __fmul_rn(vb, denom), w = __fmul_rn(vc, denom);
    v3 const q = p - fma3(ac, w, fma3(ab, v, a));
    return dot(q, q);
}

// The state of one distance query between node visits (see ray_lane).
struct distance_lane {
    v3 q;
    float best; // squared distance bound
    std::uint32_t qi, node, st_nodes, st_tris;
    int sp;
    bool touched; // a triangle touches the query: distance 0 is final
};

// Evaluates a leaf range; sets `touched` once a triangle touches the query.
template <bool Stats>
__device__ __forceinline__ void distance_leaf(spatial_params const &p, distance_lane &L, std::uint64_t r) {
    std::uint32_t const cnt = ref_count(r);
    std::uint64_t const off = ref_offset(r);
    for (std::uint32_t k = 0; k < cnt; ++k) {
        std::uint64_t const t = off + k;
        if (t >= p.primitive_count)
            continue;
        v3 a, b, c;
        record_vertices(p.tri48, t, a, b, c);
        float const d2 = point_triangle_d2(L.q, a, b, c);
        if constexpr (Stats)
            ++L.st_tris;
        if (d2 < L.best)
            L.best = d2;
    }
    L.touched = !(L.best > 0.0f);
}

// One node of detail/gwn_query_distance_impl.cuh:40-160 for L.node: children within the bound
// sorted near first, leaf children inside the node, internal children far to near with the
// nearest entered directly. s_stack is this thread's column of a [p.stack_cap][blockDim.x]
// shared-memory stack of internal node indices. False once the query is finished.
template <bool Stats>
__device__ __forceinline__ bool distance_visit(spatial_params const &p, distance_lane &L, std::uint32_t *s_stack,
                                               bool &overflow) {
    unsigned const stride = blockDim.x;
    if constexpr (Stats)
        ++L.st_nodes;
    float4 const *nd = p.nodes + static_cast<std::uint64_t>(L.node) * 8;
    cand4 cd;
    int cnt = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        float4 const A = __ldg(nd + 2 * s);
        float4 const B = __ldg(nd + 2 * s + 1);
        std::uint64_t const ref = (static_cast<std::uint64_t>(__float_as_uint(B.w)) << 32) | __float_as_uint(B.z);
        if (!ref_valid(ref))
            continue;
        float const d2 = aabb_d2(L.q, A, B);
        if (d2 >= L.best)
            continue;
        cd.put(cnt, d2, child_payload(ref, s, p.node_count));
        ++cnt;
    }
    cd.sort(cnt);
    // leaf children inside the node, near first
#pragma unroll
    for (int s = 0; s < 4; ++s)
        if (s < cnt && !L.touched && cd.pay[s] != k_invalid_u32 && (cd.pay[s] & k_leaf_payload) && cd.key[s] < L.best)
            distance_leaf<Stats>(p, L, child_ref(nd, static_cast<int>(cd.pay[s] & 3u)));
    if (L.touched)
        return false;
    // internal children far to near; the nearest is entered directly
    std::uint32_t next = k_invalid_u32;
#pragma unroll
    for (int s = 3; s >= 0; --s) {
        std::uint32_t const v = cd.pay[s];
        if (s >= cnt || overflow || v == k_invalid_u32 || (v & k_leaf_payload) || cd.key[s] >= L.best)
            continue;
        if (next != k_invalid_u32) {
            if (L.sp >= p.stack_cap) {
                overflow = true;
                continue;
            }
            s_stack[static_cast<unsigned>(L.sp) * stride] = next;
            ++L.sp;
        }
        next = v;
    }
    if (overflow)
        return false;
    if (next != k_invalid_u32) {
        L.node = next;
        return true;
    }
    if (L.sp == 0)
        return false;
    --L.sp;
    L.node = s_stack[static_cast<unsigned>(L.sp) * stride];
    return true;
}

// Loads query idx (sorted position); false when it needs no traversal (leaf root evaluated here,
// or an unusable root).
template <bool Stats>
__device__ __forceinline__ bool distance_begin(spatial_params const &p, std::uint64_t idx, distance_lane &L) {
    L.qi = p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx);
    L.q = v3{p.qx[L.qi], p.qy[L.qi], p.qz[L.qi]};
    float const band = (p.culling_band < 0.0f) ? 0.0f : p.culling_band;
    L.best = __fmul_rn(band, band);
    L.st_nodes = 0;
    L.st_tris = 0;
    L.sp = 0;
    L.touched = false;
    if (ref_leaf(p.root_ref)) {
        distance_leaf<Stats>(p, L, p.root_ref);
        return false;
    }
    if (!ref_internal(p.root_ref) || ref_offset(p.root_ref) >= p.node_count)
        return false;
    L.node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
    return true;
}

template <bool Stats>
__device__ __forceinline__ void distance_finish(spatial_params const &p, distance_lane const &L, bool overflow) {
    float result;
    if (overflow) {
        atomicOr(p.status, k_err_stack_overflow);
        result = __int_as_float(0x7fc00000);
    } else {
        result = L.touched ? 0.0f : __fsqrt_rn(L.best);
    }
    p.distance[L.qi] = result;
    if constexpr (Stats) {
        p.stat_nodes[L.qi] = L.st_nodes;
        p.stat_tris[L.qi] = L.st_tris;
    }
}

// ---- ray first hit --------------------------------------------------------------------------------

// detail/gwn_query_ray_impl.cuh:63-81: reciprocal direction with parallel axes flagged, plus
// -o * inv per axis so that each slab bound is one fused lo * inv - o * inv.
struct ray_dir {
    float inv[3], noi[3];
    bool zero[3];
};

// detail/gwn_query_ray_impl.cuh:84-139 and :259-271: closed slab test against [t_min, t_max]
// (std::min / std::max operand order, axes folded x, y, z; a parallel axis is a containment test).
// The running best never drops below t_min, so the interval is never empty on entry.
template <bool AnyZero>
__device__ __forceinline__ bool ray_box(v3 o, ray_dir const &rd, float4 A, float4 B, float t_min, float t_max,
                                        float &t_near_out) {
    float const org[3] = {o.x, o.y, o.z};
    float const lo[3] = {A.x, A.y, A.z};
    float const hi[3] = {A.w, B.x, B.y};
    float t_near = t_min, t_far = t_max;
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (AnyZero && rd.zero[k]) {
            inside = inside && (org[k] >= lo[k] && org[k] <= hi[k]);
            continue;
        }
        float const t0 = __fmaf_rn(lo[k], rd.inv[k], rd.noi[k]);
        float const t1 = __fmaf_rn(hi[k], rd.inv[k], rd.noi[k]);
        t_near = rmax(t_near, rmin(t0, t1));
        t_far = rmin(t_far, rmax(t0, t1));
    }
    t_near_out = t_near;
    return inside && t_near <= t_far;
}

// detail/gwn_query_ray_impl.cuh:142-171: component-wise stable cross products.
__device__ __forceinline__ v3 stable_normal(v3 a, v3 b, v3 c) {
    float const abx = __fmul_rn(a.z, b.y), aby = __fmul_rn(a.x, b.z), abz = __fmul_rn(a.y, b.x);
    float const bcx = __fmul_rn(b.z, c.y), bcy = __fmul_rn(b.x, c.z), bcz = __fmul_rn(b.y, c.x);
    v3 n{__fmaf_rn(b.y, c.z, -bcx), __fmaf_rn(b.z, c.x, -bcy), __fmaf_rn(b.x, c.y, -bcz)};
    if (fabsf(abx) < fabsf(bcx))
        n.x = __fmaf_rn(a.y, b.z, -abx);
    if (fabsf(aby) < fabsf(bcy))
        n.y = __fmaf_rn(a.z, b.x, -aby);
    if (fabsf(abz) < fabsf(bcz))
        n.z = __fmaf_rn(a.x, b.y, -abz);
    return n;
}

// detail/gwn_query_ray_impl.cuh:174-238: oriented Pluecker edge functions, t from the stable
// geometric normal.
__device__ __forceinline__ bool ray_triangle(v3 o, v3 d, v3 v0, v3 v1, v3 v2, float t_min, float t_max, float &t_out,
                                             float &u_out, float &v_out, v3 &n_out) {
    v3 const p0 = v0 - o, p1 = v1 - o, p2 = v2 - o;
    v3 const e0 = p2 - p0, e1 = p0 - p1, e2 = p1 - p2;
    float const u = dot(cross(e0, p2 + p0), d);
    float const v = dot(cross(e1, p0 + p1), d);
    float const w = dot(cross(e2, p1 + p2), d);
    float const uvw = __fadd_rn(__fadd_rn(u, v), w);
    float const eps = __fmul_rn(FLT_EPSILON, fabsf(uvw));
    float const mn = rmin(u, rmin(v, w));
    float const mx = rmax(u, rmax(v, w));
    if (!(mn >= -eps || mx <= eps))
        return false;
    v3 const ng = stable_normal(e0, e1, e2);
    float const den = __fmul_rn(2.0f, dot(ng, d));
    if (den == 0.0f)
        return false;
    float const t = __fdiv_rn(__fmul_rn(2.0f, dot(p0, ng)), den);
    if (!(t_min <= t && t <= t_max))
        return false;
    if (fabsf(uvw) >= FLT_MIN) {
        float const inv = __fdiv_rn(1.0f, uvw);
        u_out = __fmul_rn(u, inv);
        v_out = __fmul_rn(v, inv);
    } else {
        if (uvw == 0.0f)
            return false;
        u_out = __fdiv_rn(u, uvw);
        v_out = __fdiv_rn(v, uvw);
    }
    t_out = t;
    n_out = ng;
    return true;
}

// Canonical traversal of one ray (detail/gwn_query_ray_impl.cuh:376-560) with the best hit so far.
struct ray_best {
    float t, u, v;
    v3 n;
    std::uint32_t id;
    bool found;
};

// The state of one ray between node visits, so that a lane can hold a ray across the steps of a
// persistent loop and take another when it finishes.
struct ray_lane {
    v3 o, d;
    ray_dir rd;
    ray_best best;
    std::uint32_t qi, node, st_nodes, st_tris;
    int sp;
    bool any_zero;
};

// A leaf range against the ray: a candidate replaces the best hit when nearer, or equally near with
// a lower primitive id.
template <bool Stats>
__device__ __forceinline__ void ray_leaf(spatial_params const &p, ray_lane &L, std::uint64_t r) {
    std::uint32_t const cnt = ref_count(r);
    std::uint64_t const off = ref_offset(r);
    for (std::uint32_t k = 0; k < cnt; ++k) {
        std::uint64_t const t = off + k;
        if (t >= p.primitive_count)
            continue;
        v3 a, b, c, n;
        record_vertices(p.tri48, t, a, b, c);
        float th, uh, vh;
        if constexpr (Stats)
            ++L.st_tris;
        if (!ray_triangle(L.o, L.d, a, b, c, p.t_min, L.best.t, th, uh, vh, n))
            continue;
        std::uint32_t const id = __ldg(p.primitive_indices + t);
        if (L.best.found && !(th < L.best.t || (th == L.best.t && id < L.best.id)))
            continue;
        L.best = ray_best{th, uh, vh, n, id, true};
    }
}

// Visits L.node: the node's children against the ray (sorted near first), its leaf children, its
// internal children onto the stack far to near with the nearest taken next. False once the ray is
// finished (stack empty, or `overflow` set).
template <bool Stats, bool AnyZero>
__device__ __forceinline__ bool ray_visit(spatial_params const &p, ray_lane &L, std::uint32_t *s_stack,
                                          bool &overflow) {
    unsigned const stride = blockDim.x;
    if constexpr (Stats)
        ++L.st_nodes;
    float4 const *nd = p.nodes + static_cast<std::uint64_t>(L.node) * 8;
    cand4 cd;
    int cnt = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        float4 const A = __ldg(nd + 2 * s);
        float4 const B = __ldg(nd + 2 * s + 1);
        std::uint64_t const ref = (static_cast<std::uint64_t>(__float_as_uint(B.w)) << 32) | __float_as_uint(B.z);
        if (!ref_valid(ref))
            continue;
        float tn;
        if (!ray_box<AnyZero>(L.o, L.rd, A, B, p.t_min, L.best.t, tn))
            continue;
        cd.put(cnt, tn, child_payload(ref, s, p.node_count));
        ++cnt;
    }
    cd.sort(cnt);
#pragma unroll
    for (int s = 0; s < 4; ++s)
        if (s < cnt && cd.pay[s] != k_invalid_u32 && (cd.pay[s] & k_leaf_payload) && cd.key[s] <= L.best.t)
            ray_leaf<Stats>(p, L, child_ref(nd, static_cast<int>(cd.pay[s] & 3u)));
    std::uint32_t next = k_invalid_u32;
#pragma unroll
    for (int s = 3; s >= 0; --s) {
        std::uint32_t const v = cd.pay[s];
        if (s >= cnt || overflow || v == k_invalid_u32 || (v & k_leaf_payload) || cd.key[s] > L.best.t)
            continue;
        if (next != k_invalid_u32) {
            if (L.sp >= p.stack_cap) {
                overflow = true;
                continue;
            }
            s_stack[static_cast<unsigned>(L.sp) * stride] = next;
            ++L.sp;
        }
        next = v;
    }
    if (overflow)
        return false;
    if (next != k_invalid_u32) {
        L.node = next;
        return true;
    }
    if (L.sp == 0)
        return false;
    --L.sp;
    L.node = s_stack[static_cast<unsigned>(L.sp) * stride];
    return true;
}

template <bool Stats>
__device__ __forceinline__ bool ray_step(spatial_params const &p, ray_lane &L, std::uint32_t *s_stack,
                                         bool &overflow) {
    // parallel axes are rare: the common slab test has no per-axis branch
    return L.any_zero ? ray_visit<Stats, true>(p, L, s_stack, overflow)
                      : ray_visit<Stats, false>(p, L, s_stack, overflow);
}

// Loads ray idx (sorted position) into L. False when the ray needs no traversal: a zero direction,
// a leaf root (evaluated here) or an unusable root; L then holds the final result.
template <bool Stats>
__device__ __forceinline__ bool ray_begin(spatial_params const &p, std::uint64_t idx, ray_lane &L) {
    L.qi = p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx);
    L.o = v3{p.qx[L.qi], p.qy[L.qi], p.qz[L.qi]};
    L.d = v3{p.dx[L.qi], p.dy[L.qi], p.dz[L.qi]};
    L.st_nodes = 0;
    L.st_tris = 0;
    L.sp = 0;
    L.best = ray_best{p.t_max, 0.0f, 0.0f, v3{0.0f, 0.0f, 0.0f}, k_invalid_u32, false};
    if (!(dot(L.d, L.d) > 0.0f))
        return false;
    float const ov[3] = {L.o.x, L.o.y, L.o.z};
    float const dv[3] = {L.d.x, L.d.y, L.d.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        L.rd.zero[k] = dv[k] == 0.0f;
        L.rd.inv[k] = L.rd.zero[k] ? 0.0f : __fdiv_rn(1.0f, dv[k]);
        L.rd.noi[k] = -__fmul_rn(ov[k], L.rd.inv[k]);
    }
    L.any_zero = L.rd.zero[0] || L.rd.zero[1] || L.rd.zero[2];
    if (ref_leaf(p.root_ref)) {
        ray_leaf<Stats>(p, L, p.root_ref);
        return false;
    }
    if (!ref_internal(p.root_ref) || ref_offset(p.root_ref) >= p.node_count)
        return false;
    L.node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
    return true;
}

// Writes the ray's hit record (and statistics) at its input position.
template <bool Stats>
__device__ __forceinline__ void ray_finish(spatial_params const &p, ray_lane const &L, bool overflow) {
    if (overflow)
        atomicOr(p.status, k_err_stack_overflow);
    ray_best const &best = L.best;
    std::uint32_t const qi = L.qi;
    // miss record: t = -1, invalid id, zero weights and normal
    std::uint32_t const status = overflow ? GWNB_RAY_OVERFLOW : (best.found ? GWNB_RAY_HIT : GWNB_RAY_MISS);
    float4 const lo = best.found ? make_float4(best.t, best.u, best.v, best.n.x) : make_float4(-1.0f, 0.0f, 0.0f, 0.0f);
    float4 const hi = best.found ? make_float4(best.n.y, best.n.z, __uint_as_float(best.id), __uint_as_float(status))
                                 : make_float4(0.0f, 0.0f, __uint_as_float(k_invalid_u32), __uint_as_float(status));
    if ((reinterpret_cast<std::uintptr_t>(p.hits) & 15u) == 0u) {
        float4 *out = reinterpret_cast<float4 *>(p.hits + qi);
        out[0] = lo;
        out[1] = hi;
    } else { // caller storage aligned to 4 bytes only
        float *out = reinterpret_cast<float *>(p.hits + qi);
        out[0] = lo.x;
        out[1] = lo.y;
        out[2] = lo.z;
        out[3] = lo.w;
        out[4] = hi.x;
        out[5] = hi.y;
        out[6] = hi.z;
        out[7] = hi.w;
    }
    if constexpr (Stats) {
        p.stat_nodes[qi] = L.st_nodes;
        p.stat_tris[qi] = L.st_tris;
    }
}

// Query positions claimed per warp at a time by the persistent kernels (consecutive sorted
// positions, so the queries a warp holds stay within one neighbourhood -- and, for rays, one
// direction cell).
constexpr unsigned k_refill_chunk = 64;

struct ray_walk {
    using lane = ray_lane;
    template <bool Stats> static __device__ __forceinline__ bool begin(spatial_params const &p, std::uint64_t i, lane &L) {
        return ray_begin<Stats>(p, i, L);
    }
    template <bool Stats>
    static __device__ __forceinline__ bool step(spatial_params const &p, lane &L, std::uint32_t *col, bool &overflow) {
        return ray_step<Stats>(p, L, col, overflow);
    }
    template <bool Stats> static __device__ __forceinline__ void finish(spatial_params const &p, lane const &L, bool o) {
        ray_finish<Stats>(p, L, o);
    }
};

struct distance_walk {
    using lane = distance_lane;
    template <bool Stats> static __device__ __forceinline__ bool begin(spatial_params const &p, std::uint64_t i, lane &L) {
        return distance_begin<Stats>(p, i, L);
    }
    template <bool Stats>
    static __device__ __forceinline__ bool step(spatial_params const &p, lane &L, std::uint32_t *col, bool &overflow) {
        return distance_visit<Stats>(p, L, col, overflow);
    }
    template <bool Stats> static __device__ __forceinline__ void finish(spatial_params const &p, lane const &L, bool o) {
        distance_finish<Stats>(p, L, o);
    }
};

// Persistent batch: each lane walks its own query one node per step, and a lane whose query has
// finished takes the warp's next unclaimed query before the next step, instead of idling until
// the warp's longest traversal ends (sorted rays on the 1M-triangle sphere: 18 nodes on average,
// 41 for a warp's longest). Each query's traversal, and so its result and statistics, is the
// per-query canonical one. Every lane of every warp runs the loop to the end (the ballots take all
// lanes). 10M rays: 10.4 ms sorted and 9.3 ms in input order, against 11.8 and 14.7 ms one ray per
// thread.
template <class W, bool Stats> __device__ __forceinline__ void walk(spatial_params const &p, std::uint32_t *col) {
    unsigned const lane = threadIdx.x & 31u;
    unsigned const below = (1u << lane) - 1u;
    std::uint64_t chunk_next = 0, chunk_end = 0;
    bool drained = false, have = false, overflow = false;
    typename W::lane L;
    for (;;) {
        unsigned need = __ballot_sync(0xffffffffu, !have);
        while (need != 0u && !drained) {
            if (chunk_next >= chunk_end) {
                unsigned long long base = 0;
                if (lane == 0)
                    base = atomicAdd(p.next_item, static_cast<unsigned long long>(k_refill_chunk));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= p.n) {
                    drained = true;
                    break;
                }
                chunk_next = base;
                chunk_end = base + k_refill_chunk < p.n ? base + k_refill_chunk : p.n;
            }
            std::uint64_t const avail = chunk_end - chunk_next;
            unsigned const want = static_cast<unsigned>(__popc(need));
            unsigned const take = avail < want ? static_cast<unsigned>(avail) : want;
            unsigned const rank = static_cast<unsigned>(__popc(need & below));
            if (((need >> lane) & 1u) != 0u && rank < take) {
                overflow = false;
                have = W::template begin<Stats>(p, chunk_next + rank, L);
                if (!have)
                    W::template finish<Stats>(p, L, false);
            }
            chunk_next += take;
            need = __ballot_sync(0xffffffffu, !have);
        }
        if (__ballot_sync(0xffffffffu, have) == 0u)
            break;
        if (have && !W::template step<Stats>(p, L, col, overflow)) {
            W::template finish<Stats>(p, L, overflow);
            have = false;
        }
    }
}

// The shared-memory stack holds exactly the BVH's internal stack bound per thread.
template <bool Stats> __global__ void __launch_bounds__(256) k_ray(spatial_params p) {
    extern __shared__ std::uint32_t s_stack[]; // [p.stack_cap][blockDim.x]
    walk<ray_walk, Stats>(p, s_stack + threadIdx.x);
}

// Distance queries in Hilbert order stay one per thread: a warp's traversals are similar enough
// that refilling lanes costs as much coherence as it saves (10M queries on the 1M-triangle sphere:
// 96 ms one per thread, 100 ms persistent). Queries in input order take the persistent form
// (k_distance_walk: 104 ms against 291 ms one per thread).
template <bool Stats> __global__ void __launch_bounds__(256) k_distance(spatial_params p) {
    extern __shared__ std::uint32_t s_stack[]; // [p.stack_cap][blockDim.x]
    std::uint64_t const idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= p.n)
        return;
    distance_lane L;
    bool overflow = false;
    if (distance_begin<Stats>(p, idx, L))
        while (distance_visit<Stats>(p, L, s_stack + threadIdx.x, overflow)) {
        }
    distance_finish<Stats>(p, L, overflow);
}

// Warp-cooperative distance walk for batches in Hilbert order: the 32 lanes of a warp (32
// neighbouring queries) walk one traversal together. Every stack entry carries the mask of lanes
// that still need the subtree; at a node each lane tests the four child boxes against its own
// bound, the leaf children are evaluated by the lanes that need them (slot order) and the internal
// ones are pushed far to near by the smallest box distance among the lanes that need them, the
// nearest entered directly. A lane leaves a subtree when the child box is no nearer than its bound
// and leaves the walk once a triangle touches it. Each lane's result is the minimum over the
// triangles its own pruning lets through -- the same triangle set bound as the per-thread walk, so
// the same minimum -- only the order of the visits differs (and with it how soon a bound tightens).
// The stack lives in the lanes' registers (entry e in lane e & 31, bank e >> 5), as in the Taylor
// warp walk; the union walk never holds more entries than the tree's internal stack bound.
template <int Cap> __global__ void __launch_bounds__(256) k_distance_warp(spatial_params p) {
    static_assert(Cap <= 64, "warp stack holds at most 64 entries");
    unsigned const lane = threadIdx.x & 31u;
    std::uint64_t const idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool const valid = idx < p.n;
    if (__ballot_sync(0xffffffffu, valid) == 0u)
        return;
    distance_lane L{};
    bool const walks = valid && distance_begin<false>(p, idx, L);
    unsigned mask = __ballot_sync(0xffffffffu, walks);
    bool overflow = false;
    if (mask != 0u) {
        std::uint32_t node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
        std::uint32_t st_node0 = 0, st_node1 = 0;
        unsigned st_mask0 = 0, st_mask1 = 0;
        int sp = 0;
        for (;;) {
            mask &= __ballot_sync(0xffffffffu, walks && !L.touched);
            if (mask != 0u && node < p.node_count) {
                bool const active = ((mask >> lane) & 1u) != 0u;
                float4 const *nd = p.nodes + static_cast<std::uint64_t>(node) * 8;
                // internal children that some lane needs: (warp-nearest box distance, node, lanes)
                std::uint32_t key[4], child[4];
                unsigned cm[4];
                int ni = 0;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    key[s] = 0xffffffffu;
                    child[s] = k_invalid_u32;
                    cm[s] = 0u;
                }
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    float4 const A = __ldg(nd + 2 * s);
                    float4 const B = __ldg(nd + 2 * s + 1);
                    std::uint64_t const ref =
                        (static_cast<std::uint64_t>(__float_as_uint(B.w)) << 32) | __float_as_uint(B.z);
                    if (!ref_valid(ref))
                        continue;
                    float const d2 = active ? aabb_d2(L.q, A, B) : 0.0f;
                    bool const want = active && d2 < L.best;
                    unsigned const m = __ballot_sync(0xffffffffu, want);
                    if (m == 0u)
                        continue;
                    if (ref_leaf(ref)) {
                        if (want && !L.touched && d2 < L.best)
                            distance_leaf<false>(p, L, ref);
                    } else if (ref_offset(ref) < p.node_count) {
                        // d2 >= 0, so its bits order like the value
                        std::uint32_t const k = __reduce_min_sync(0xffffffffu, want ? __float_as_uint(d2) : 0xffffffffu);
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if (j == ni) {
                                key[j] = k;
                                child[j] = static_cast<std::uint32_t>(ref_offset(ref));
                                cm[j] = m;
                            }
                        ++ni;
                    }
                }
                // near first (the five-comparator network on the uniform keys)
                auto cswap = [&](int l, int r) {
                    if (key[l] > key[r]) {
                        std::uint32_t const tk = key[l], tc = child[l];
                        unsigned const tm = cm[l];
                        key[l] = key[r];
                        child[l] = child[r];
                        cm[l] = cm[r];
                        key[r] = tk;
                        child[r] = tc;
                        cm[r] = tm;
                    }
                };
                cswap(0, 1);
                cswap(2, 3);
                cswap(0, 2);
                cswap(1, 3);
                cswap(1, 2);
                std::uint32_t next = k_invalid_u32;
                unsigned next_mask = 0u;
#pragma unroll
                for (int s = 3; s >= 0; --s) {
                    if (child[s] == k_invalid_u32)
                        continue;
                    if (next != k_invalid_u32) {
                        if (sp >= Cap || sp >= p.stack_cap) {
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
                    next = child[s];
                    next_mask = cm[s];
                }
                if (overflow)
                    break;
                if (next != k_invalid_u32) {
                    node = next;
                    mask = next_mask;
                    continue;
                }
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
    if (valid)
        distance_finish<false>(p, L, walks && overflow);
}

template <bool Stats> __global__ void __launch_bounds__(256) k_distance_walk(spatial_params p) {
    extern __shared__ std::uint32_t s_stack[]; // [p.stack_cap][blockDim.x]
    walk<distance_walk, Stats>(p, s_stack + threadIdx.x);
}

// ---- ray ordering ---------------------------------------------------------------------------------

// Direction bits of the ray sort key (even; half per octahedral axis).
#ifndef GWNB_RAY_DIR_BITS
#define GWNB_RAY_DIR_BITS 6
#endif
constexpr int k_ray_dir_bits = GWNB_RAY_DIR_BITS;
static_assert(k_ray_dir_bits % 2 == 0 && k_ray_dir_bits <= 16, "direction bits: even, at most 16");

// 30-bit sort key of a ray: the cell of its direction on the octahedral map of the unit sphere
// (k_ray_dir_bits bits, Morton order of the two map coordinates) above the leading bits of its
// origin's Hilbert index, so that the 32 rays of a warp share a direction cone and a neighbourhood
// and walk similar paths. Rays with a zero or NaN direction land in cell 0.
__global__ void __launch_bounds__(256)
    k_ray_codes(float const *__restrict__ ox, float const *__restrict__ oy, float const *__restrict__ oz,
                float const *__restrict__ dx, float const *__restrict__ dy, float const *__restrict__ dz,
                std::uint64_t n, aabb const *__restrict__ root, std::uint32_t *__restrict__ codes) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    std::uint32_t const h = hilbert_code30(*root, ox[i], oy[i], oz[i]);
    if constexpr (k_ray_dir_bits == 0) {
        codes[i] = h;
        return;
    }
    float const x = dx[i], y = dy[i], z = dz[i];
    float const l1 = fabsf(x) + fabsf(y) + fabsf(z);
    float u = 0.0f, v = 0.0f;
    if (l1 > 0.0f) {
        u = x / l1;
        v = y / l1;
        if (z < 0.0f) { // fold the lower hemisphere onto the corners of the square
            float const fu = (1.0f - fabsf(v)) * (u >= 0.0f ? 1.0f : -1.0f);
            v = (1.0f - fabsf(u)) * (v >= 0.0f ? 1.0f : -1.0f);
            u = fu;
        }
    }
    constexpr int b = k_ray_dir_bits / 2;
    constexpr float cells = static_cast<float>(1u << b);
    auto cell = [&](float f) -> std::uint32_t {
        f = fminf(fmaxf(f * 0.5f + 0.5f, 0.0f), 1.0f); // NaN -> 0
        return min(static_cast<std::uint32_t>(f * cells), (1u << b) - 1u);
    };
    std::uint32_t const cu = cell(u), cv = cell(v);
    std::uint32_t dir = 0;
#pragma unroll
    for (int k = 0; k < b; ++k)
        dir |= (((cu >> k) & 1u) << (2 * k + 1)) | (((cv >> k) & 1u) << (2 * k));
    codes[i] = (dir << (30 - k_ray_dir_bits)) | (h >> k_ray_dir_bits);
}

// ---- host launchers ----------------------------------------------------------------------------------

template <class Kern> int launch_per_query(Kern kern, spatial_params const &p, int block, cudaStream_t s) {
    std::size_t const smem = static_cast<std::size_t>(p.stack_cap) * block * sizeof(std::uint32_t);
    if (smem > 48 * 1024)
        GWNB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    unsigned const grid = static_cast<unsigned>((p.n + block - 1) / block);
    note_launch(), kern<<<grid, block, smem, s>>>(p);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

// A persistent grid (resident blocks per SM x SMs, fewer for a small batch) whose warps claim
// queries through a counter zeroed on the stream before the launch.
template <class Kern> int launch_persistent(Kern kern, spatial_params p, int block, cudaStream_t s) {
    std::size_t const smem = static_cast<std::size_t>(p.stack_cap) * block * sizeof(std::uint32_t);
    if (smem > 48 * 1024)
        GWNB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int per_sm = 0;
    GWNB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem));
    if (per_sm < 1)
        per_sm = 1;
    std::uint64_t const needed = (p.n + block - 1) / block;
    std::uint64_t const resident = static_cast<std::uint64_t>(device_sm_count()) * static_cast<std::uint64_t>(per_sm);
    unsigned const grid = static_cast<unsigned>(needed < resident ? needed : resident);
    GWNB_TRY(alloc(&p.next_item, 1, s));
    cudaError_t e = cudaMemsetAsync(p.next_item, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        note_launch(), kern<<<grid, block, smem, s>>>(p);
        e = cudaGetLastError();
    }
    release(p.next_item, s);
    if (e != cudaSuccess)
        return set_cuda_error(e, "persistent spatial kernel");
    return GWNB_OK;
}

template <int Cap> int launch_distance_warp(spatial_params const &p, cudaStream_t s) {
    unsigned const grid = static_cast<unsigned>((p.n + 255) / 256);
    note_launch(), k_distance_warp<Cap><<<grid, 256, 0, s>>>(p);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

// warp_walk: a distance batch in Hilbert order walked warp-cooperatively (k_distance_warp).
template <bool Ray, bool Stats> int launch_spatial(spatial_params const &p, int block, bool warp_walk, cudaStream_t s) {
    if (Ray)
        return launch_persistent(k_ray<Stats>, p, block, s);
    if (warp_walk)
        return p.stack_cap <= 32 ? launch_distance_warp<32>(p, s) : launch_distance_warp<64>(p, s);
    return p.order != nullptr ? launch_per_query(k_distance<Stats>, p, block, s)
                              : launch_persistent(k_distance_walk<Stats>, p, block, s);
}

// Sort order of a ray batch by the key of k_ray_codes: order[i] is the index of the i-th ray.
int ray_order(bvh_aux_impl const *a, float const *ox, float const *oy, float const *oz, float const *dx,
              float const *dy, float const *dz, std::uint64_t n, std::uint32_t *order, cudaStream_t s) {
    if (n == 0)
        return GWNB_OK;
    std::uint32_t *codes = nullptr, *sorted = nullptr;
    int rc = alloc(&codes, n, s);
    if (rc == GWNB_OK)
        rc = alloc(&sorted, n, s);
    if (rc == GWNB_OK) {
        note_launch(), k_ray_codes<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(ox, oy, oz, dx, dy, dz, n, a->root_bounds,
                                                                          codes);
        rc = radix_sort_pairs(codes, sorted, nullptr, order, n, 4, 30, s, a->status);
    }
    release(codes, s);
    release(sorted, s);
    return rc;
}

struct spatial_request {
    bool ray;
    float const *qx, *qy, *qz, *dx, *dy, *dz;
    float *distance;
    ray_hit *hits;
    std::uint32_t *stat_nodes, *stat_tris;
    std::uint64_t n;
    float culling_band, t_min, t_max;
    gwnb_spatial_options opt;
};

int spatial_batch(gwnb_bvh4_f32 *b, spatial_request const &r, cudaStream_t s) {
    if (r.n == 0)
        return GWNB_OK;
    GWNB_TRY(ensure_bvh_aux(b, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    spatial_params p{};
    p.nodes = reinterpret_cast<float4 const *>(b->nodes);
    p.node_count = b->node_count;
    p.tri48 = a->tri48;
    p.primitive_indices = b->primitive_indices;
    p.primitive_count = b->primitive_count;
    p.root_ref = b->root.reference;
    p.qx = r.qx;
    p.qy = r.qy;
    p.qz = r.qz;
    p.dx = r.dx;
    p.dy = r.dy;
    p.dz = r.dz;
    p.distance = r.distance;
    p.hits = r.hits;
    p.stat_nodes = r.stat_nodes;
    p.stat_tris = r.stat_tris;
    p.n = r.n;
    p.culling_band = r.culling_band;
    p.t_min = r.t_min;
    p.t_max = r.t_max;
    p.status = a->status;
    std::uint32_t *order = nullptr;
    if (r.opt.sort_queries != 0 && r.n > 1) {
        GWNB_TRY(alloc(&order, r.n, s));
        int const rc = r.ray ? ray_order(a, r.qx, r.qy, r.qz, r.dx, r.dy, r.dz, r.n, order, s)
                             : query_order(a->root_bounds, r.qx, r.qy, r.qz, r.n, order, s, a->status);
        if (rc != GWNB_OK) {
            release(order, s);
            return rc;
        }
        p.order = order;
    }
    // the traversal never holds more than the internal stack bound (validated against the capacity)
    p.stack_cap = ref_internal(b->root.reference) ? static_cast<int>(b->internal_stack_bound) : 0;
    if (p.stack_cap < 1)
        p.stack_cap = 1;
    bool const stats = r.stat_nodes != nullptr;
    // the walk of a distance batch in Hilbert order (the statistics keep the per-thread walk, whose
    // visit counts are the canonical traversal's)
    walk_plan plan;
    plan.per_thread = true;
    if (!r.ray && !stats && p.order != nullptr && p.stack_cap <= 64) {
        plan.per_thread = r.opt.per_thread == GWNB_WALK_THREAD;
        if (r.opt.per_thread == GWNB_WALK_TIMED) {
            int device = 0;
            (void)cudaGetDevice(&device);
            float const band = r.culling_band;
            std::uint32_t band_bits = 0;
            std::memcpy(&band_bits, &band, sizeof(band_bits));
            int size_class = 0;
            for (std::uint64_t v = r.n; v > 1; v >>= 1)
                ++size_class;
            plan = plan_walk(walk_kind{b->nodes, device, 1, 0, 0, 0, 1, size_class, band_bits}, s);
        }
    }
    if (plan.start != nullptr)
        (void)cudaEventRecord(plan.start, s);
    int const block = query_launch_block(r.opt.block_size);
    bool const warp = !plan.per_thread;
    int rc;
    if (r.ray)
        rc = stats ? launch_spatial<true, true>(p, block, false, s) : launch_spatial<true, false>(p, block, false, s);
    else
        rc = stats ? launch_spatial<false, true>(p, block, false, s) : launch_spatial<false, false>(p, block, warp, s);
    if (plan.stop != nullptr)
        (void)cudaEventRecord(plan.stop, s);
    release(order, s);
    return rc;
}

// Shared validation in smallgwn's order (include/gwn/gwn_query.cuh:149-170 and :232-248).
int spatial_options(gwnb_bvh4_f32 const *b, gwnb_spatial_options const *in, gwnb_spatial_options &o) {
    o = gwnb_spatial_options{256, 64, 0, GWNB_WALK_WARP};
    if (in != nullptr) {
        o = *in;
        if (o.block_size == 0)
            o.block_size = 256;
        if (o.stack_capacity == 0)
            o.stack_capacity = 64;
    }
    if (o.block_size < 32 || o.block_size > 1024 || (o.block_size % 32) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch block size must be a multiple of 32 in [32, 1024].");
    if (o.stack_capacity <= 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity must be positive.");
    if (o.per_thread < GWNB_WALK_WARP || o.per_thread > GWNB_WALK_TIMED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown traversal (per_thread must be 0, 1 or 2).");
    if (ref_internal(b->root.reference) && b->internal_stack_bound > static_cast<std::uint32_t>(o.stack_capacity))
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity is below the BVH internal stack bound.");
    // the shared-memory stack holds the internal stack bound for every thread of a block
    if (ref_internal(b->root.reference) &&
        static_cast<std::uint64_t>(b->internal_stack_bound) * query_launch_block(o.block_size) *
                sizeof(std::uint32_t) >
            227u * 1024u)
        return set_error(GWNB_INVALID_ARGUMENT,
                         "Traversal stack bound times block size exceeds the 227 KB of shared memory per block.");
    // candidate payloads hold internal node indices below 2^31 (the top bit marks leaves)
    if (b->node_count >= 0x80000000ull)
        return set_error(GWNB_INVALID_ARGUMENT, "BVH node count exceeds 2^31 - 1.");
    return GWNB_OK;
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_unsigned_distance_batch_f32(const gwnb_bvh4_f32 *b, const float *qx, const float *qy, const float *qz,
                                     float *out, uint64_t n, float culling_band, const gwnb_spatial_options *opt,
                                     gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_unsigned_distance");
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    gwnb_spatial_options o;
    GWNB_TRY(spatial_options(b, opt, o));
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) || !has_storage(out, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    if (n == 0)
        return GWNB_OK;
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    spatial_request r{};
    r.ray = false;
    r.qx = qx;
    r.qy = qy;
    r.qz = qz;
    r.distance = out;
    r.n = n;
    r.culling_band = culling_band;
    r.opt = o;
    return spatial_batch(const_cast<gwnb_bvh4_f32 *>(b), r, as_cuda(stream));
} catch (...) {
    return host_exception();
}

int gwnb_ray_first_hit_batch_f32(const gwnb_bvh4_f32 *b, const float *ox, const float *oy, const float *oz,
                                 const float *dx, const float *dy, const float *dz, gwnb_ray_hit_f32 *out, uint64_t n,
                                 float t_min, float t_max, const gwnb_spatial_options *opt, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_ray_first_hit");
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    gwnb_spatial_options o;
    GWNB_TRY(spatial_options(b, opt, o));
    if (!has_storage(ox, n) || !has_storage(oy, n) || !has_storage(oz, n) || !has_storage(dx, n) ||
        !has_storage(dy, n) || !has_storage(dz, n) || !has_storage(out, n))
        return set_error(GWNB_INVALID_ARGUMENT,
                         "ray first-hit: ray/output spans must use non-null storage when non-empty.");
    if (!(t_max >= t_min))
        return set_error(GWNB_INVALID_ARGUMENT, "ray first-hit: requires t_max >= t_min.");
    if (n == 0)
        return GWNB_OK;
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    spatial_request r{};
    r.ray = true;
    r.qx = ox;
    r.qy = oy;
    r.qz = oz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    r.hits = reinterpret_cast<ray_hit *>(out);
    r.n = n;
    r.t_min = t_min;
    r.t_max = t_max;
    r.opt = o;
    return spatial_batch(const_cast<gwnb_bvh4_f32 *>(b), r, as_cuda(stream));
} catch (...) {
    return host_exception();
}

int gwnb_spatial_stats_f32(const gwnb_bvh4_f32 *b, int kind, const float *qx, const float *qy, const float *qz,
                           const float *dx, const float *dy, const float *dz, uint64_t n, float culling_band,
                           float t_min, float t_max, uint32_t *nodes_entered, uint32_t *triangles_tested,
                           gwnb_stream_t stream) try {
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (kind != GWNB_SPATIAL_DISTANCE && kind != GWNB_SPATIAL_RAY)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown spatial query kind.");
    gwnb_spatial_options const want{256, 128, 0};
    gwnb_spatial_options o;
    GWNB_TRY(spatial_options(b, &want, o));
    bool const ray = kind == GWNB_SPATIAL_RAY;
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) || !has_storage(nodes_entered, n) ||
        !has_storage(triangles_tested, n) ||
        (ray && (!has_storage(dx, n) || !has_storage(dy, n) || !has_storage(dz, n))))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    if (ray && !(t_max >= t_min))
        return set_error(GWNB_INVALID_ARGUMENT, "ray first-hit: requires t_max >= t_min.");
    if (n == 0)
        return GWNB_OK;
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    cudaStream_t const s = as_cuda(stream);
    spatial_request r{};
    r.ray = ray;
    r.qx = qx;
    r.qy = qy;
    r.qz = qz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    r.n = n;
    r.culling_band = culling_band;
    r.t_min = t_min;
    r.t_max = t_max;
    r.stat_nodes = nodes_entered;
    r.stat_tris = triangles_tested;
    r.opt = o;
    // the results themselves go to scratch
    float *dist = nullptr;
    ray_hit *hits = nullptr;
    if (ray) {
        GWNB_TRY(alloc(&hits, n, s));
        r.hits = hits;
    } else {
        GWNB_TRY(alloc(&dist, n, s));
        r.distance = dist;
    }
    int const rc = spatial_batch(const_cast<gwnb_bvh4_f32 *>(b), r, s);
    release(hits, s);
    release(dist, s);
    return rc;
} catch (...) {
    return host_exception();
}

int gwnb_ray_order_f32(const gwnb_bvh4_f32 *b_in, const float *ox, const float *oy, const float *oz,
                       const float *dx, const float *dy, const float *dz, uint64_t n, uint32_t *order,
                       gwnb_stream_t stream) try {
    if (!bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (!has_storage(ox, n) || !has_storage(oy, n) || !has_storage(oz, n) || !has_storage(dx, n) ||
        !has_storage(dy, n) || !has_storage(dz, n) || !has_storage(order, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    return ray_order(reinterpret_cast<bvh_aux_impl const *>(b->aux), ox, oy, oz, dx, dy, dz, n, order, s);
} catch (...) {
    return host_exception();
}

} // extern "C"
