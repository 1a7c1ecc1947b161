// Boundary chains and antipodal winding numbers.
//
// smallgwn: include/gwn/gwn_boundary.cuh:20-129 and detail/gwn_boundary_impl.cuh:34-415 (the
// algebraic boundary of the oriented triangle chain), include/gwn/gwn_query.cuh:446-656 and
// detail/gwn_query_winding_antipodal_impl.cuh:54-602 (the antipodal method of Martens, Trettner
// and Bessmeltsev, ACM TOG 45(4), 2026: signed crossings of a coordinate ray plus a spherical-area
// term over the boundary chain, axes +z, +x, +y tried in turn until neither term is singular).
//
// Boundary chain: one 64-bit key (low vertex << b | high vertex, b bits per vertex index) per
// triangle edge with its orientation, one stable radix sort (2b key bits instead of two full
// 32-bit passes), a segmented sum per key, and an ordered compaction by block counts and a scan;
// rows come out in ascending (low, high) order as in smallgwn.
//
// Antipodal batch: one thread per query (optionally in Hilbert order), the crossings by a
// canonical traversal of the BVH4 with the stack in shared memory, the boundary term from
// per-call edge records (both end points and the multiplicity, 32 bytes, read with warp-uniform
// addresses) summed in FP64. Arithmetic is rounded operation by operation with dot products,
// cross products and determinants fused in one fixed pattern that the oracle restates with fmaf;
// the FP64 running sum replaces smallgwn's Kahan sum in float. Stack overflow writes NaN and sets
// the BVH's device error bit instead of trapping.
#include "gwnb_internal.cuh"

#include <algorithm>

namespace gwnb {

int query_order(aabb const *root_bounds, float const *qx, float const *qy, float const *qz, std::uint64_t n,
                std::uint32_t *order, cudaStream_t s, unsigned int *status);

namespace {

constexpr double k_pi_d = 3.141592653589793238462643383279502884;

// ---- boundary chain ---------------------------------------------------------------------------------

// detail/gwn_boundary_impl.cuh:34-60: three keyed edges per triangle, orientation +1 low -> high,
// -1 high -> low, 0 for a degenerate edge (stored as orientation + 1).
__global__ void __launch_bounds__(256)
    k_edge_keys(std::uint32_t const *__restrict__ i0, std::uint32_t const *__restrict__ i1,
                std::uint32_t const *__restrict__ i2, std::uint64_t nt, std::uint64_t nv, int bits,
                std::uint64_t *__restrict__ keys, std::uint32_t *__restrict__ orient, unsigned int *bad_index) {
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= nt)
        return;
    std::uint32_t const v[3] = {i0[t], i1[t], i2[t]};
    if (v[0] >= nv || v[1] >= nv || v[2] >= nv)
        atomicOr(bad_index, 1u);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        std::uint32_t const a = v[k], b = v[(k + 1) % 3];
        std::uint32_t const lo = min(a, b), hi = max(a, b);
        keys[t * 3 + k] = (static_cast<std::uint64_t>(lo) << bits) | hi;
        orient[t * 3 + k] = a < b ? 2u : (b < a ? 0u : 1u);
    }
}

// Net orientation of the key group starting at i, 0 unless i heads its group.
__device__ __forceinline__ int group_sum(std::uint64_t const *keys, std::uint32_t const *orient, std::uint64_t n,
                                         std::uint64_t i) {
    if (i > 0 && keys[i] == keys[i - 1])
        return 0;
    int sum = static_cast<int>(orient[i]) - 1;
    for (std::uint64_t j = i + 1; j < n && keys[j] == keys[i]; ++j)
        sum += static_cast<int>(orient[j]) - 1;
    return sum;
}

constexpr int k_chain_block = 256;

// detail/gwn_boundary_impl.cuh:127-171: a row per group head with nonzero net orientation; here the
// per-block row counts of the ordered compaction.
__global__ void __launch_bounds__(k_chain_block)
    k_chain_count(std::uint64_t const *__restrict__ keys, std::uint32_t const *__restrict__ orient, std::uint64_t n,
                  std::uint32_t *__restrict__ block_rows) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool const row = i < n && group_sum(keys, orient, n, i) != 0;
    std::uint32_t const c = __syncthreads_count(row);
    if (threadIdx.x == 0)
        block_rows[blockIdx.x] = c;
}

// Exclusive scan of the block counts in place (one block; the last slot receives the total).
__global__ void __launch_bounds__(1024) k_chain_scan(std::uint32_t *__restrict__ counts, std::uint64_t blocks) {
    __shared__ unsigned long long s_carry;
    __shared__ unsigned long long s_warp[32];
    if (threadIdx.x == 0)
        s_carry = 0;
    __syncthreads();
    unsigned const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (std::uint64_t base = 0; base < blocks + 1; base += blockDim.x) {
        std::uint64_t const i = base + threadIdx.x;
        unsigned long long v = i < blocks ? counts[i] : 0ull;
        unsigned long long x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            unsigned long long const y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= static_cast<unsigned>(d))
                x += y;
        }
        if (lane == 31)
            s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = lane < blockDim.x / 32 ? s_warp[lane] : 0ull;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                unsigned long long const y = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= static_cast<unsigned>(d))
                    w += y;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        unsigned long long const warp_base = warp > 0 ? s_warp[warp - 1] : 0ull;
        unsigned long long const excl = s_carry + warp_base + x - v;
        if (i <= blocks)
            counts[i] = static_cast<std::uint32_t>(excl);
        __syncthreads();
        if (threadIdx.x == 0)
            s_carry += s_warp[blockDim.x / 32 - 1];
        __syncthreads();
    }
}

// Ordered emission: block offset plus the rank of the row inside its block.
__global__ void __launch_bounds__(k_chain_block)
    k_chain_emit(std::uint64_t const *__restrict__ keys, std::uint32_t const *__restrict__ orient, std::uint64_t n,
                 int bits, std::uint32_t const *__restrict__ block_offsets, std::uint32_t *__restrict__ start,
                 std::uint32_t *__restrict__ end, std::uint64_t *__restrict__ mult) {
    __shared__ std::uint32_t s_warp[k_chain_block / 32];
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    int const sum = i < n ? group_sum(keys, orient, n, i) : 0;
    bool const row = sum != 0;
    unsigned const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned const ballot = __ballot_sync(0xffffffffu, row);
    if (lane == 0)
        s_warp[warp] = __popc(ballot);
    __syncthreads();
    std::uint32_t before = 0;
    for (unsigned w = 0; w < warp; ++w)
        before += s_warp[w];
    if (!row)
        return;
    std::uint32_t const out = block_offsets[blockIdx.x] + before + __popc(ballot & ((1u << lane) - 1u));
    std::uint32_t const lo = static_cast<std::uint32_t>(keys[i] >> bits);
    std::uint32_t const hi = static_cast<std::uint32_t>(keys[i] & ((std::uint64_t(1) << bits) - 1u));
    start[out] = sum > 0 ? lo : hi;
    end[out] = sum > 0 ? hi : lo;
    mult[out] = static_cast<std::uint64_t>(sum > 0 ? sum : -sum);
}

// ---- antipodal arithmetic (same fused pattern as the oracle) -------------------------------------

struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 sub3(v3 a, v3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ v3 add3(v3 a, v3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ v3 scale3(v3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ v3 fma3(v3 a, float s, v3 c) {
    return {__fmaf_rn(a.x, s, c.x), __fmaf_rn(a.y, s, c.y), __fmaf_rn(a.z, s, c.z)};
}
__device__ __forceinline__ float dot3(v3 a, v3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ float dop(float a, float b, float c, float d) { return __fmaf_rn(a, b, -__fmul_rn(c, d)); }
__device__ __forceinline__ v3 cross3(v3 a, v3 b) {
    return {dop(a.y, b.z, a.z, b.y), dop(a.z, b.x, a.x, b.z), dop(a.x, b.y, a.y, b.x)};
}

// Projection orthogonal to the ray axis (:54-63): x -> (y, z), y -> (z, x), z -> (x, y).
template <int Axis> __device__ __forceinline__ float proj_u(v3 v) { return Axis == 0 ? v.y : (Axis == 1 ? v.z : v.x); }
template <int Axis> __device__ __forceinline__ float proj_v(v3 v) { return Axis == 0 ? v.z : (Axis == 1 ? v.x : v.y); }
template <int Axis> __device__ __forceinline__ float along(v3 v) { return Axis == 0 ? v.x : (Axis == 1 ? v.y : v.z); }

__device__ __forceinline__ int sign_of(float v) { return v > 0.0f ? 1 : (v < 0.0f ? -1 : 0); }

// :76-111: projected determinant, its sign under the lexicographic symbolic perturbation, and the
// singular flag of a collinear edge whose end points lie on opposite sides of the query.
template <int Axis> struct edge_class {
    float det;
    int sign;
    bool singular;
};
template <int Axis> __device__ __forceinline__ edge_class<Axis> classify(v3 s, v3 e) {
    float const ax = proj_u<Axis>(s), ay = proj_v<Axis>(s), bx = proj_u<Axis>(e), by = proj_v<Axis>(e);
    float const d = dop(ax, by, ay, bx);
    int sg = sign_of(d);
    if (sg == 0) {
        sg = sign_of(__fsub_rn(ay, by));
        if (sg == 0)
            sg = sign_of(__fsub_rn(bx, ax));
    }
    bool const singular = d == 0.0f && __fmaf_rn(ay, by, __fmul_rn(ax, bx)) <= 0.0f;
    return {d, sg, singular};
}

// :123-177: crossing of one oriented triangle with the positive axis ray from q; false when singular.
template <int Axis> __device__ __forceinline__ bool triangle_crossing(v3 q, v3 a, v3 b, v3 c, float &sum) {
    v3 const pa = sub3(a, q), pb = sub3(b, q), pc = sub3(c, q);
    v3 const n = cross3(sub3(pb, pa), sub3(pc, pa));
    float const na = along<Axis>(n);
    if (na == 0.0f)
        return true;
    edge_class<Axis> const e0 = classify<Axis>(pa, pb), e1 = classify<Axis>(pb, pc), e2 = classify<Axis>(pc, pa);
    if (e0.singular || e1.singular || e2.singular)
        return false;
    if (e0.sign == 0 || e1.sign == 0 || e2.sign == 0)
        return false;
    if (!((e0.sign >= 0 && e1.sign >= 0 && e2.sign >= 0) || (e0.sign <= 0 && e1.sign <= 0 && e2.sign <= 0)))
        return true;
    float const t = __fdiv_rn(dot3(n, pa), na);
    if (t == 0.0f)
        return false;
    if (!(t > 0.0f))
        return true;
    sum += na > 0.0f ? 1.0f : -1.0f;
    return true;
}

struct antipodal_params {
    float4 const *nodes; // node_count x 8 float4
    std::uint64_t node_count;
    triangle48 const *tri48;
    std::uint64_t primitive_count;
    std::uint64_t root_ref;
    float4 const *edges; // 2 float4 per boundary row: (start, multiplicity), (end, 0)
    std::uint64_t edge_count;
    float const *qx, *qy, *qz;
    std::uint32_t const *order;
    float *out;
    float *gx, *gy, *gz;
    std::uint64_t n;
    int stack_cap;
    unsigned int *status;
};

// Vertices of a padded record, v0 + e (as every BVH query here reconstructs them).
__device__ __forceinline__ void tri_vertices(triangle48 const *t48, std::uint64_t i, v3 &a, v3 &b, v3 &c) {
    float4 const A = __ldg(&t48[i].a);
    float4 const B = __ldg(&t48[i].b);
    float4 const C = __ldg(&t48[i].c);
    a = {A.x, A.y, A.z};
    b = add3(a, v3{A.w, B.x, B.y});
    c = add3(a, v3{B.z, B.w, C.x});
}

// :380-489: signed crossings of the positive axis ray through the canonical BVH (children in slot
// order, leaves evaluated in place, the last internal child entered directly). 0 done, 1 singular,
// 2 stack overflow.
template <int Axis>
__device__ __forceinline__ int crossings(antipodal_params const &p, v3 q, std::uint32_t *s_stack, float &sum) {
    constexpr int U = Axis == 0 ? 1 : (Axis == 1 ? 2 : 0);
    constexpr int W = Axis == 0 ? 2 : (Axis == 1 ? 0 : 1);
    float const qc[3] = {q.x, q.y, q.z};
    sum = 0.0f;
    auto leaf = [&](std::uint64_t r) -> bool {
        std::uint32_t const cnt = ref_count(r);
        std::uint64_t const off = ref_offset(r);
        for (std::uint32_t k = 0; k < cnt; ++k) {
            std::uint64_t const t = off + k;
            if (t >= p.primitive_count)
                continue;
            v3 a, b, c;
            tri_vertices(p.tri48, t, a, b, c);
            if (!triangle_crossing<Axis>(q, a, b, c, sum))
                return false;
        }
        return true;
    };
    if (ref_leaf(p.root_ref))
        return leaf(p.root_ref) ? 0 : 1;
    unsigned const stride = blockDim.x;
    int sp = 0;
    std::uint64_t node = ref_offset(p.root_ref);
    for (;;) {
        std::uint64_t next = ~std::uint64_t(0);
        if (node < p.node_count) {
            float4 const *nd = p.nodes + node * 8;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                float4 const A = __ldg(nd + 2 * s);
                float4 const B = __ldg(nd + 2 * s + 1);
                std::uint64_t const r = (static_cast<std::uint64_t>(__float_as_uint(B.w)) << 32) | __float_as_uint(B.z);
                if (!ref_valid(r))
                    continue;
                float const lo[3] = {A.x, A.y, A.z}, hi[3] = {A.w, B.x, B.y};
                if (!(qc[U] >= lo[U] && qc[U] <= hi[U] && qc[W] >= lo[W] && qc[W] <= hi[W] && hi[Axis] >= qc[Axis]))
                    continue;
                if (ref_leaf(r)) {
                    if (!leaf(r))
                        return 1;
                    continue;
                }
                if (!ref_internal(r))
                    continue;
                if (next != ~std::uint64_t(0)) {
                    if (sp >= p.stack_cap)
                        return 2;
                    s_stack[static_cast<unsigned>(sp) * stride] = static_cast<std::uint32_t>(next);
                    ++sp;
                }
                next = ref_offset(r);
            }
        }
        if (next != ~std::uint64_t(0)) {
            node = next;
            continue;
        }
        if (sp == 0)
            return 0;
        --sp;
        node = s_stack[static_cast<unsigned>(sp) * stride];
    }
}

// Terms whose atan2 arguments are both below 1/16 of |s||e| are guarded: the edge passes close to the
// ray line seen from the query, where float rounding dominates the arguments and the gradient term
// (which grows like the inverse of that distance) cancels against its neighbours. Their atan2
// arguments are recomputed in FP64 (the angle itself is then well conditioned) and their gradient
// evaluated in FP64. The decision is taken on the float values, exactly as the oracle takes it.
constexpr float k_ap_guard2 = 1.0f / 256.0f;

struct area_args {
    float ls, le, num, den;
};

template <int Axis> __device__ __forceinline__ v3 minus_ray() {
    return {Axis == 0 ? -1.0f : 0.0f, Axis == 1 ? -1.0f : 0.0f, Axis == 2 ? -1.0f : 0.0f};
}

// :188-205: |s|, |e| and the atan2 arguments of the signed spherical area of (-ray, s, e).
template <int Axis> __device__ __forceinline__ area_args area_arguments(v3 s, v3 e, float det) {
    v3 const mr = minus_ray<Axis>();
    area_args r;
    r.ls = __fsqrt_rn(dot3(s, s));
    r.le = __fsqrt_rn(dot3(e, e));
    r.num = -det;
    if (det == 0.0f)
        r.num = dot3(mr, cross3(s, e));
    r.den = __fmaf_rn(dot3(e, mr), r.ls, __fadd_rn(__fmaf_rn(dot3(mr, s), r.le, __fmul_rn(r.ls, r.le)), dot3(s, e)));
    return r;
}

__device__ __forceinline__ bool guarded(area_args const &a) {
    float const sl = __fmul_rn(a.ls, a.le);
    return __fmaf_rn(a.den, a.den, __fmul_rn(a.num, a.num)) < __fmul_rn(k_ap_guard2, __fmul_rn(sl, sl));
}

// FP64 vectors, |s|, |e| and atan2 arguments of a guarded term, from the float end points and query.
struct area_args_d {
    double s[3], e[3], ls, le, num, den;
};
template <int Axis> __device__ __forceinline__ area_args_d area_arguments_d(float4 A, float4 B, v3 q) {
    area_args_d r;
    r.s[0] = static_cast<double>(A.x) - q.x;
    r.s[1] = static_cast<double>(A.y) - q.y;
    r.s[2] = static_cast<double>(A.z) - q.z;
    r.e[0] = static_cast<double>(B.x) - q.x;
    r.e[1] = static_cast<double>(B.y) - q.y;
    r.e[2] = static_cast<double>(B.z) - q.z;
    double const c[3] = {r.s[1] * r.e[2] - r.s[2] * r.e[1], r.s[2] * r.e[0] - r.s[0] * r.e[2],
                         r.s[0] * r.e[1] - r.s[1] * r.e[0]};
    r.ls = sqrt(r.s[0] * r.s[0] + r.s[1] * r.s[1] + r.s[2] * r.s[2]);
    r.le = sqrt(r.e[0] * r.e[0] + r.e[1] * r.e[1] + r.e[2] * r.e[2]);
    r.num = -c[Axis];
    r.den = r.ls * r.le - r.s[Axis] * r.le - r.e[Axis] * r.ls + (r.s[0] * r.e[0] + r.s[1] * r.e[1] + r.s[2] * r.e[2]);
    return r;
}

// One boundary row against query q: the end points relative to q.
__device__ __forceinline__ void row_ends(float4 A, float4 B, v3 q, v3 &s, v3 &e) {
    s = {__fsub_rn(A.x, q.x), __fsub_rn(A.y, q.y), __fsub_rn(A.z, q.z)};
    e = {__fsub_rn(B.x, q.x), __fsub_rn(B.y, q.y), __fsub_rn(B.z, q.z)};
}

// :221-249: the term of one boundary row for one axis: multiplicity times the signed spherical area
// (on the positive branch for the x and y axes), the atan2 arguments of guarded terms from FP64
// vectors; false when the row is singular.
template <int Axis> __device__ __forceinline__ bool row_term(float4 A, float4 B, v3 q, double &term) {
    v3 s, e;
    row_ends(A, B, q, s, e);
    edge_class<Axis> const c = classify<Axis>(s, e);
    if (c.singular)
        return false;
    area_args const a = area_arguments<Axis>(s, e, c.det);
    if (!(a.ls > 0.0f) || !(a.le > 0.0f)) {
        term = __longlong_as_double(0x7ff8000000000000ll);
        return true;
    }
    float num = a.num, den = a.den;
    if (guarded(a)) { // accurately known arguments leave the angle well conditioned: atan2 in float
        area_args_d const d = area_arguments_d<Axis>(A, B, q);
        num = static_cast<float>(d.num);
        den = static_cast<float>(d.den);
    }
    float area = __fmul_rn(2.0f, atan2f(num, den));
    if (Axis != 2 && c.sign > 0 && area < 0.0f)
        area = __fadd_rn(area, static_cast<float>(2.0 * k_pi_d));
    term = static_cast<double>(__fmul_rn(A.w, area));
    return true;
}

// :209-256: boundary term of one axis (FP64 sum in row order); false when singular.
template <int Axis> __device__ __forceinline__ bool boundary_term(antipodal_params const &p, v3 q, double &out) {
    double sum = 0.0;
    for (std::uint64_t i = 0; i < p.edge_count; ++i) {
        double term;
        if (!row_term<Axis>(__ldg(p.edges + 2 * i), __ldg(p.edges + 2 * i + 1), q, term))
            return false;
        sum += term;
    }
    out = sum / (4.0 * k_pi_d);
    return true;
}

// Crossings plus boundary term of one axis for one query. 0 done, 1 singular, 2 overflow.
template <int Axis> __device__ __forceinline__ int antipodal_axis(antipodal_params const &p, v3 q, std::uint32_t *s_stack,
                                                                 float &result) {
    float cross;
    int const c = crossings<Axis>(p, q, s_stack, cross);
    if (c != 0)
        return c;
    double b;
    if (!boundary_term<Axis>(p, q, b))
        return 1;
    result = static_cast<float>(static_cast<double>(cross) + b);
    return 0;
}

// Value batch (:533-568): k_ap_q queries per thread. The +z axis, which decides almost every query,
// runs for the whole block together: crossings per thread, then the boundary rows in tiles of
// k_ap_tile staged in shared memory and shared by all queries of the block. A query whose +z
// crossings or boundary rows are singular retries +x and +y on its own (global loads). One query
// per thread fits 60 registers (4 resident blocks of 256) where two took 80 (3 blocks): 11 % less
// time on 1M queries against 2,048 boundary rows, results bit-identical.
constexpr int k_ap_tile = 256;
constexpr int k_ap_q = 1;

__global__ void __launch_bounds__(256) k_antipodal(antipodal_params p) {
    extern __shared__ float4 s_dyn[]; // [2 * k_ap_tile] edge tile, then [p.stack_cap][blockDim.x] stack
    float4 *s_rows = s_dyn;
    std::uint32_t *s_stack = reinterpret_cast<std::uint32_t *>(s_dyn + 2 * k_ap_tile) + threadIdx.x;
    std::uint64_t const base_idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x * k_ap_q + threadIdx.x;
    std::uint32_t qi[k_ap_q];
    v3 q[k_ap_q];
    float cross[k_ap_q];
    int rc[k_ap_q]; // 0 done so far, 1 singular on +z, 2 overflow, 3 no query
    double sum[k_ap_q];
#pragma unroll
    for (int k = 0; k < k_ap_q; ++k) {
        std::uint64_t const idx = base_idx + static_cast<std::uint64_t>(k) * blockDim.x;
        sum[k] = 0.0;
        cross[k] = 0.0f;
        if (idx >= p.n) {
            rc[k] = 3;
            qi[k] = 0;
            q[k] = {0.0f, 0.0f, 0.0f};
            continue;
        }
        qi[k] = p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx);
        q[k] = {p.qx[qi[k]], p.qy[qi[k]], p.qz[qi[k]]};
        rc[k] = crossings<2>(p, q[k], s_stack, cross[k]);
    }
    for (std::uint64_t base = 0; base < p.edge_count; base += k_ap_tile) {
        int const cnt = static_cast<int>(p.edge_count - base < k_ap_tile ? p.edge_count - base : k_ap_tile);
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * cnt; t += blockDim.x)
            s_rows[t] = __ldg(p.edges + 2 * base + t);
        __syncthreads();
        // four rows in flight: their square roots and atan2 interleave (the FP64 sum still adds
        // the terms in row order); 2-4 % less time, results bit-identical
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            float4 const A = s_rows[2 * j], B = s_rows[2 * j + 1];
#pragma unroll
            for (int k = 0; k < k_ap_q; ++k) {
                if (rc[k] != 0)
                    continue;
                double term;
                if (row_term<2>(A, B, q[k], term))
                    sum[k] += term;
                else
                    rc[k] = 1;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < k_ap_q; ++k) {
        if (rc[k] == 3)
            continue;
        float result = __int_as_float(0x7fc00000);
        int r = rc[k];
        if (r == 0)
            result = static_cast<float>(static_cast<double>(cross[k]) + sum[k] / (4.0 * k_pi_d));
        if (r == 1)
            r = antipodal_axis<0>(p, q[k], s_stack, result);
        if (r == 1)
            r = antipodal_axis<1>(p, q[k], s_stack, result);
        if (r == 2)
            atomicOr(p.status, k_err_stack_overflow);
        if (r != 0)
            result = __int_as_float(0x7fc00000);
        p.out[qi[k]] = result;
    }
}

// :261-304: gradient of one signed spherical-area term with respect to the query (float).
template <int Axis> __device__ __forceinline__ v3 area_gradient(v3 s, v3 e, area_args const &a) {
    float const nan = __int_as_float(0x7fc00000);
    v3 const mr = minus_ray<Axis>();
    if (a.ls == 0.0f || a.le == 0.0f)
        return {nan, nan, nan};
    v3 const su = scale3(s, __fdiv_rn(1.0f, a.ls)), eu = scale3(e, __fdiv_rn(1.0f, a.le));
    float const d2 = __fmaf_rn(a.den, a.den, __fmul_rn(a.num, a.num));
    if (d2 == 0.0f)
        return {nan, nan, nan};
    float const cn = __fdiv_rn(__fmul_rn(2.0f, a.den), d2), cd = __fdiv_rn(__fmul_rn(-2.0f, a.num), d2);
    v3 const gn = scale3(add3(cross3(e, mr), cross3(mr, s)), -1.0f);
    v3 const t1 = scale3(fma3(su, __fadd_rn(1.0f, dot3(mr, eu)), add3(mr, eu)), a.le);
    v3 const t2 = scale3(fma3(eu, __fadd_rn(1.0f, dot3(mr, su)), add3(mr, su)), a.ls);
    v3 const gd = scale3(add3(t1, t2), -1.0f);
    return fma3(gd, cd, scale3(gn, cn));
}

// The same gradient in FP64 for a guarded term.
template <int Axis> __device__ __forceinline__ void area_gradient_d(area_args_d const &d, double g[3]) {
    double const nan = __longlong_as_double(0x7ff8000000000000ll);
    double const d2 = d.num * d.num + d.den * d.den;
    if (d.ls == 0.0 || d.le == 0.0 || d2 == 0.0) {
        g[0] = g[1] = g[2] = nan;
        return;
    }
    double mr[3] = {0.0, 0.0, 0.0};
    mr[Axis] = -1.0;
    double su[3], eu[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        su[k] = d.s[k] / d.ls;
        eu[k] = d.e[k] / d.le;
    }
    double const cn = 2.0 * d.den / d2, cd = -2.0 * d.num / d2;
    double const me = -eu[Axis], ms = -su[Axis];
    double const gn[3] = {-((d.e[1] * mr[2] - d.e[2] * mr[1]) + (mr[1] * d.s[2] - mr[2] * d.s[1])),
                          -((d.e[2] * mr[0] - d.e[0] * mr[2]) + (mr[2] * d.s[0] - mr[0] * d.s[2])),
                          -((d.e[0] * mr[1] - d.e[1] * mr[0]) + (mr[0] * d.s[1] - mr[1] * d.s[0]))};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double const t1 = d.le * (mr[k] + eu[k] + (1.0 + me) * su[k]);
        double const t2 = d.ls * (mr[k] + su[k] + (1.0 + ms) * eu[k]);
        g[k] = cn * gn[k] - cd * (t1 + t2);
    }
}

// :320-332: the gradient term of one boundary row for one axis (multiplicity times the area
// gradient, float or guarded FP64); false when singular.
template <int Axis> __device__ __forceinline__ bool row_gradient(float4 A, float4 B, v3 q, double term[3]) {
    v3 s, e;
    row_ends(A, B, q, s, e);
    edge_class<Axis> const c = classify<Axis>(s, e);
    if (c.singular)
        return false;
    area_args const a = area_arguments<Axis>(s, e, c.det);
    if (a.ls != 0.0f && a.le != 0.0f && guarded(a)) {
        double g[3];
        area_gradient_d<Axis>(area_arguments_d<Axis>(A, B, q), g);
        double const m = static_cast<double>(A.w);
        term[0] = m * g[0];
        term[1] = m * g[1];
        term[2] = m * g[2];
        return true;
    }
    v3 const g = area_gradient<Axis>(s, e, a);
    term[0] = static_cast<double>(__fmul_rn(A.w, g.x));
    term[1] = static_cast<double>(__fmul_rn(A.w, g.y));
    term[2] = static_cast<double>(__fmul_rn(A.w, g.z));
    return true;
}

// :307-334: gradient of the boundary term of one axis (FP64 sums); false when singular.
template <int Axis> __device__ __forceinline__ bool boundary_gradient(antipodal_params const &p, v3 q, v3 &out) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (std::uint64_t i = 0; i < p.edge_count; ++i) {
        double t[3];
        if (!row_gradient<Axis>(__ldg(p.edges + 2 * i), __ldg(p.edges + 2 * i + 1), q, t))
            return false;
        sx += t[0];
        sy += t[1];
        sz += t[2];
    }
    double const k4 = 4.0 * k_pi_d;
    out = {static_cast<float>(sx / k4), static_cast<float>(sy / k4), static_cast<float>(sz / k4)};
    return true;
}

// Gradient batch (:336-372), tiled like the value batch on the +z axis, one query per thread.
__global__ void __launch_bounds__(256) k_antipodal_gradient(antipodal_params p) {
    __shared__ float4 s_rows[2 * k_ap_tile];
    std::uint64_t const idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool const valid = idx < p.n;
    std::uint32_t const qi = valid ? (p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx)) : 0u;
    v3 const q = valid ? v3{p.qx[qi], p.qy[qi], p.qz[qi]} : v3{0.0f, 0.0f, 0.0f};
    bool ok = valid;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (std::uint64_t base = 0; base < p.edge_count; base += k_ap_tile) {
        int const cnt = static_cast<int>(p.edge_count - base < k_ap_tile ? p.edge_count - base : k_ap_tile);
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * cnt; t += blockDim.x)
            s_rows[t] = __ldg(p.edges + 2 * base + t);
        __syncthreads();
        for (int j = 0; j < cnt && ok; ++j) {
            double t[3];
            if (row_gradient<2>(s_rows[2 * j], s_rows[2 * j + 1], q, t)) {
                sx += t[0];
                sy += t[1];
                sz += t[2];
            } else {
                ok = false;
            }
        }
    }
    if (!valid)
        return;
    float const nan = __int_as_float(0x7fc00000);
    v3 g{nan, nan, nan};
    double const k4 = 4.0 * k_pi_d;
    if (ok)
        g = {static_cast<float>(sx / k4), static_cast<float>(sy / k4), static_cast<float>(sz / k4)};
    else if (!boundary_gradient<0>(p, q, g) && !boundary_gradient<1>(p, q, g))
        g = {nan, nan, nan};
    p.gx[qi] = g.x;
    p.gy[qi] = g.y;
    p.gz[qi] = g.z;
}

// Edge records of the chain over the current positions: (start, multiplicity), (end, 0).
__global__ void __launch_bounds__(256)
    k_edge_records(gwnb_geometry_f32 g, std::uint32_t const *__restrict__ start, std::uint32_t const *__restrict__ end,
                   std::uint64_t const *__restrict__ mult, std::uint64_t n, float4 *__restrict__ out) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    std::uint32_t const a = start[i], b = end[i];
    bool const ok = a < g.vertex_count && b < g.vertex_count;
    float const nan = __int_as_float(0x7fc00000);
    out[2 * i] = ok ? make_float4(g.vertex_x[a], g.vertex_y[a], g.vertex_z[a], static_cast<float>(mult[i]))
                    : make_float4(nan, nan, nan, 0.0f);
    out[2 * i + 1] = ok ? make_float4(g.vertex_x[b], g.vertex_y[b], g.vertex_z[b], 0.0f) : make_float4(nan, nan, nan, 0.0f);
}

int bits_for(std::uint64_t v) {
    int b = 1;
    while (b < 32 && (std::uint64_t(1) << b) < v)
        ++b;
    return b;
}

void release_chain(gwnb_boundary_chain_u32 &c, cudaStream_t s) {
    release(c.start_vertex, s);
    release(c.end_vertex, s);
    release(c.multiplicity, s);
    c = gwnb_boundary_chain_u32{};
}

bool chain_valid(gwnb_boundary_chain_u32 const *c) {
    return c != nullptr && c->is_built != 0 &&
           (c->edge_count == 0 || (c->start_vertex != nullptr && c->end_vertex != nullptr && c->multiplicity != nullptr));
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_boundary_chain_build_u32(const gwnb_geometry_f32 *g, gwnb_boundary_chain_u32 *out, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::build_boundary_chain");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "Boundary chain output is null.");
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry object contains no queryable data.");
    cudaStream_t const s = as_cuda(stream);
    std::uint64_t const nt = g->triangle_count, nv = g->vertex_count;
    gwnb_boundary_chain_u32 staging{};
    staging.mesh_vertex_count = nv;
    staging.mesh_triangle_count = nt;
    staging.is_built = 1;
    if (nt == 0) {
        *out = staging;
        return GWNB_OK;
    }
    std::uint64_t const ne = nt * 3;
    if (ne >= (std::uint64_t(1) << 30))
        return set_error(GWNB_INVALID_ARGUMENT, "Boundary chain preprocessing supports fewer than 2^30 edges.");
    int const bits = bits_for(nv);
    std::uint64_t *keys = nullptr, *keys_sorted = nullptr;
    std::uint32_t *orient = nullptr, *orient_sorted = nullptr, *blocks = nullptr;
    unsigned int *flags = nullptr; // [0] bad index, [1] sort status
    std::uint64_t const nblocks = (ne + k_chain_block - 1) / k_chain_block;
    int rc = GWNB_OK;
    auto cleanup = [&]() {
        release(keys, s);
        release(keys_sorted, s);
        release(orient, s);
        release(orient_sorted, s);
        release(blocks, s);
        release(flags, s);
    };
    if ((rc = alloc(&keys, ne, s)) != GWNB_OK || (rc = alloc(&keys_sorted, ne, s)) != GWNB_OK ||
        (rc = alloc(&orient, ne, s)) != GWNB_OK || (rc = alloc(&orient_sorted, ne, s)) != GWNB_OK ||
        (rc = alloc(&blocks, nblocks + 1, s)) != GWNB_OK || (rc = alloc(&flags, 2, s)) != GWNB_OK) {
        cleanup();
        return rc;
    }
    cudaError_t e = cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        note_launch(), k_edge_keys<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, s>>>(g->tri_i0, g->tri_i1, g->tri_i2, nt, nv, bits,
                                                                           keys, orient, flags);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cleanup();
        return set_cuda_error(e, "boundary chain edge keys");
    }
    if ((rc = radix_sort_pairs(keys, keys_sorted, orient, orient_sorted, ne, 8, 2 * bits, s, flags + 1)) != GWNB_OK) {
        cleanup();
        return rc;
    }
    note_launch(), k_chain_count<<<static_cast<unsigned>(nblocks), k_chain_block, 0, s>>>(keys_sorted, orient_sorted, ne, blocks);
    note_launch(), k_chain_scan<<<1, 1024, 0, s>>>(blocks, nblocks);
    unsigned int host_flags[2] = {0, 0};
    std::uint32_t rows = 0;
    e = cudaMemcpyAsync(&rows, blocks + nblocks, sizeof(rows), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cleanup();
        return set_cuda_error(e, "boundary chain count");
    }
    if (host_flags[0] != 0) {
        cleanup();
        return set_error(GWNB_INVALID_ARGUMENT, "Triangle index out of range.");
    }
    if (host_flags[1] != 0) {
        cleanup();
        return set_error(GWNB_INTERNAL_ERROR, "boundary chain: radix sort look-back timed out.");
    }
    staging.edge_count = rows;
    if (rows > 0) {
        if ((rc = alloc(&staging.start_vertex, rows, s)) != GWNB_OK || (rc = alloc(&staging.end_vertex, rows, s)) != GWNB_OK ||
            (rc = alloc(&staging.multiplicity, rows, s)) != GWNB_OK) {
            release_chain(staging, s);
            cleanup();
            return rc;
        }
        note_launch(), k_chain_emit<<<static_cast<unsigned>(nblocks), k_chain_block, 0, s>>>(
            keys_sorted, orient_sorted, ne, bits, blocks, staging.start_vertex, staging.end_vertex, staging.multiplicity);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            release_chain(staging, s);
            cleanup();
            return set_cuda_error(e, "boundary chain emit");
        }
    }
    cleanup();
    *out = staging;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

void gwnb_boundary_chain_release_u32(gwnb_boundary_chain_u32 *chain, gwnb_stream_t stream) {
    if (chain != nullptr)
        release_chain(*chain, as_cuda(stream));
}

static int antipodal_common(const gwnb_geometry_f32 *g, const gwnb_bvh4_f32 *b_in, const gwnb_boundary_chain_u32 *c,
                            const float *qx, const float *qy, const float *qz, float *out, float *gx, float *gy,
                            float *gz, uint64_t n, const gwnb_spatial_options *opt, gwnb_stream_t stream) {
    bool const gradient = gx != nullptr || gy != nullptr || gz != nullptr;
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry object contains no queryable data.");
    gwnb_spatial_options o{256, 64, 0};
    if (opt != nullptr) {
        o = *opt;
        if (o.block_size == 0)
            o.block_size = 256;
        if (o.stack_capacity == 0)
            o.stack_capacity = 64;
    }
    if (o.block_size < 32 || o.block_size > 1024 || (o.block_size % 32) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch block size must be a multiple of 32 in [32, 1024].");
    if (!gradient) {
        if (!bvh_valid(b_in))
            return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
        if (b_in->primitive_count != g->triangle_count)
            return set_error(GWNB_INVALID_ARGUMENT, "Geometry and BVH triangle counts differ.");
        if (o.stack_capacity <= 0)
            return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity must be positive.");
        if (ref_internal(b_in->root.reference) && b_in->internal_stack_bound > static_cast<std::uint32_t>(o.stack_capacity))
            return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity is below the BVH internal stack bound.");
        if (ref_internal(b_in->root.reference) &&
            static_cast<std::uint64_t>(b_in->internal_stack_bound) * query_launch_block(o.block_size) * 4u +
                    2u * k_ap_tile * 16u >
                227u * 1024u)
            return set_error(GWNB_INVALID_ARGUMENT,
                             "Traversal stack bound times block size exceeds the 227 KB of shared memory per block.");
        if (b_in->node_count >= 0x80000000ull)
            return set_error(GWNB_INVALID_ARGUMENT, "BVH node count exceeds 2^31 - 1.");
    }
    if (!chain_valid(c))
        return set_error(GWNB_INVALID_ARGUMENT, "Boundary chain object is unbuilt or invalid.");
    if (c->mesh_vertex_count != g->vertex_count || c->mesh_triangle_count != g->triangle_count)
        return set_error(GWNB_INVALID_ARGUMENT, "Boundary chain belongs to a different mesh shape.");
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) ||
        (!gradient && !has_storage(out, n)) ||
        (gradient && (!has_storage(gx, n) || !has_storage(gy, n) || !has_storage(gz, n))))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans require non-null storage when non-empty.");
    if (n == 0)
        return GWNB_OK;
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    cudaStream_t const s = as_cuda(stream);
    antipodal_params p{};
    bvh_aux_impl *a = nullptr;
    if (!gradient) {
        auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
        GWNB_TRY(ensure_bvh_aux(b, s));
        a = reinterpret_cast<bvh_aux_impl *>(b->aux);
        p.nodes = reinterpret_cast<float4 const *>(b->nodes);
        p.node_count = b->node_count;
        p.tri48 = a->tri48;
        p.primitive_count = b->primitive_count;
        p.root_ref = b->root.reference;
        p.status = a->status;
        p.stack_cap = ref_internal(b->root.reference) ? static_cast<int>(b->internal_stack_bound) : 0;
        if (p.stack_cap < 1)
            p.stack_cap = 1;
    }
    float4 *edges = nullptr;
    std::uint32_t *order = nullptr;
    int rc = GWNB_OK;
    if (c->edge_count > 0) {
        GWNB_TRY(alloc(&edges, 2 * c->edge_count, s));
        note_launch(), k_edge_records<<<static_cast<unsigned>((c->edge_count + 255) / 256), 256, 0, s>>>(
            *g, c->start_vertex, c->end_vertex, c->multiplicity, c->edge_count, edges);
    }
    if (o.sort_queries != 0 && n > 1 && a != nullptr) {
        rc = alloc(&order, n, s);
        if (rc == GWNB_OK)
            rc = query_order(a->root_bounds, qx, qy, qz, n, order, s, a->status);
    }
    if (rc == GWNB_OK) {
        p.edges = edges;
        p.edge_count = c->edge_count;
        p.qx = qx;
        p.qy = qy;
        p.qz = qz;
        p.order = order;
        p.out = out;
        p.gx = gx;
        p.gy = gy;
        p.gz = gz;
        p.n = n;
        int const block = query_launch_block(o.block_size);
        if (gradient) {
            unsigned const grid = static_cast<unsigned>((n + block - 1) / block);
            note_launch(), k_antipodal_gradient<<<grid, block, 0, s>>>(p);
        } else {
            std::uint64_t const per_block = static_cast<std::uint64_t>(block) * k_ap_q;
            unsigned const grid = static_cast<unsigned>((n + per_block - 1) / per_block);
            std::size_t const smem = 2 * k_ap_tile * sizeof(float4) +
                                     static_cast<std::size_t>(p.stack_cap) * block * sizeof(std::uint32_t);
            cudaError_t e = cudaSuccess;
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(k_antipodal, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            if (e == cudaSuccess)
                note_launch(), k_antipodal<<<grid, block, smem, s>>>(p);
        }
        cudaError_t const e = cudaGetLastError();
        if (e != cudaSuccess)
            rc = set_cuda_error(e, "antipodal batch launch");
    }
    release(edges, s);
    release(order, s);
    return rc;
}

int gwnb_winding_antipodal_batch_f32(const gwnb_geometry_f32 *g, const gwnb_bvh4_f32 *b,
                                     const gwnb_boundary_chain_u32 *chain, const float *qx, const float *qy,
                                     const float *qz, float *out, uint64_t n, const gwnb_spatial_options *options,
                                     gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_antipodal");
    return antipodal_common(g, b, chain, qx, qy, qz, out, nullptr, nullptr, nullptr, n, options, stream);
} catch (...) {
    return host_exception();
}

int gwnb_winding_gradient_antipodal_batch_f32(const gwnb_geometry_f32 *g, const gwnb_boundary_chain_u32 *chain,
                                              const float *qx, const float *qy, const float *qz, float *gx, float *gy,
                                              float *gz, uint64_t n, int block_size, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_antipodal_gradient");
    if (n > 0 && (gx == nullptr || gy == nullptr || gz == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans require non-null storage when non-empty.");
    gwnb_spatial_options const o{block_size, 64, 0};
    // a non-null marker selects the gradient path even for an empty batch
    float marker = 0.0f;
    return antipodal_common(g, nullptr, chain, qx, qy, qz, nullptr, gx ? gx : &marker, gy ? gy : &marker,
                            gz ? gz : &marker, n, &o, stream);
} catch (...) {
    return host_exception();
}

} // extern "C"
