// BVH construction kernels: scene bounds, triangle AABB + Morton codes, Karras LBVH topology,
// bottom-up binary bounds, level-synchronous BVH4 collapse and leaf-ordered triangle records.
//
// Arithmetic that decides topology follows smallgwn exactly so that Morton codes, the sorted
// permutation and the LBVH topology are bit-identical:
//   Morton: detail/gwn_bvh_build_common.cuh:22-88, :157-214 (centroid (min+max)*0.5, normalise
//           with the scene inverse extent, clamp to [0,1], scale by 1023 / 2097151, truncate,
//           interleave x<<2 | y<<1 | z);
//   scene:  :243-274 (inverse = 1 when the extent is zero);
//   Karras: detail/gwn_bvh_build_binary.cuh:29-129 (delta with the index tie-break);
//   collapse rule: detail/gwn_bvh_build_collapse.cuh:163-199 (expand the internal candidate with
//           the largest half-area, ties to the lower binary index, right child appended).
// The collapse itself is restructured: every tree level allocates its child node ids with a
// decoupled look-back scan, which yields a canonical breadth-first node order directly (no
// persistent work queue, no reorder sort). A build enqueues the first 32 levels without a host
// round trip (a level past the bottom exits at once) and learns from its single read-back whether
// the tree was deeper.
#include "gwnb_internal.cuh"

#include <algorithm>
#include <vector>

namespace gwnb {

namespace {

constexpr int k_block = 256;

__device__ inline unsigned int float_to_ordered(float f) {
    unsigned int const u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ inline float ordered_to_float(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// words[0..2] = ordered min x,y,z (init 0xffffffff), words[3..5] = ordered max (init 0).
__global__ void __launch_bounds__(k_block)
    k_scene_bounds(float const *__restrict__ x, float const *__restrict__ y,
                   float const *__restrict__ z, std::uint64_t n, unsigned int *words) {
    float mn[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float mx[3] = {-mn[0], -mn[1], -mn[2]};
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        float const v[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = rmin(mn[a], v[a]);
            mx[a] = rmax(mx[a], v[a]);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        unsigned int omn = float_to_ordered(mn[a]);
        unsigned int omx = float_to_ordered(mx[a]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            omn = min(omn, __shfl_xor_sync(0xffffffffu, omn, o));
            omx = max(omx, __shfl_xor_sync(0xffffffffu, omx, o));
        }
        if ((threadIdx.x & 31u) == 0u) {
            atomicMin(&words[a], omn);
            atomicMax(&words[3 + a], omx);
        }
    }
}

template <class K> struct morton_traits;
template <> struct morton_traits<std::uint32_t> {
    static constexpr float k_quant = 1023.0f;
    __device__ static std::uint32_t expand(std::uint32_t v) {
        std::uint32_t x = v & 0x000003ffu;
        x = (x | (x << 16)) & 0x030000ffu;
        x = (x | (x << 8)) & 0x0300f00fu;
        x = (x | (x << 4)) & 0x030c30c3u;
        x = (x | (x << 2)) & 0x09249249u;
        return x;
    }
};
template <> struct morton_traits<std::uint64_t> {
    static constexpr float k_quant = 2097151.0f;
    __device__ static std::uint64_t expand(std::uint64_t v) {
        std::uint64_t x = v & 0x1fffffull;
        x = (x | (x << 32)) & 0x1f00000000ffffull;
        x = (x | (x << 16)) & 0x1f0000ff0000ffull;
        x = (x | (x << 8)) & 0x100f00f00f00f00full;
        x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
        x = (x | (x << 2)) & 0x1249249249249249ull;
        return x;
    }
};

__device__ inline float clamp01(float v) {
    if (v < 0.0f)
        return 0.0f;
    if (v > 1.0f)
        return 1.0f;
    return v;
}

template <class K>
__global__ void __launch_bounds__(k_block)
    k_morton(gwnb_geometry_f32 g, unsigned int const *__restrict__ scene, aabb *__restrict__ aabbs,
             K *__restrict__ codes) {
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= g.triangle_count)
        return;
    float smin[3], sinv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float const lo = ordered_to_float(scene[a]);
        float const hi = ordered_to_float(scene[3 + a]);
        smin[a] = lo;
        sinv[a] = (hi == lo) ? 1.0f : __fdiv_rn(1.0f, __fsub_rn(hi, lo));
    }
    std::uint32_t const ia = g.tri_i0[t], ib = g.tri_i1[t], ic = g.tri_i2[t];
    std::uint64_t const nv = g.vertex_count;
    if (ia >= nv || ib >= nv || ic >= nv) {
        aabbs[t] = aabb{0, 0, 0, 0, 0, 0};
        codes[t] = 0;
        return;
    }
    float const ax = g.vertex_x[ia], ay = g.vertex_y[ia], az = g.vertex_z[ia];
    float const bx = g.vertex_x[ib], by = g.vertex_y[ib], bz = g.vertex_z[ib];
    float const cx = g.vertex_x[ic], cy = g.vertex_y[ic], cz = g.vertex_z[ic];
    aabb const b{rmin(ax, rmin(bx, cx)), rmin(ay, rmin(by, cy)), rmin(az, rmin(bz, cz)),
                 rmax(ax, rmax(bx, cx)), rmax(ay, rmax(by, cy)), rmax(az, rmax(bz, cz))};
    aabbs[t] = b;
    float const ctr[3] = {__fmul_rn(__fadd_rn(b.min_x, b.max_x), 0.5f),
                          __fmul_rn(__fadd_rn(b.min_y, b.max_y), 0.5f),
                          __fmul_rn(__fadd_rn(b.min_z, b.max_z), 0.5f)};
    K q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float const nrm = clamp01(__fmul_rn(__fsub_rn(ctr[a], smin[a]), sinv[a]));
        q[a] = static_cast<K>(__fmul_rn(nrm, morton_traits<K>::k_quant));
    }
    codes[t] = (morton_traits<K>::expand(q[0]) << 2) | (morton_traits<K>::expand(q[1]) << 1) |
               morton_traits<K>::expand(q[2]);
}

__global__ void __launch_bounds__(k_block)
    k_gather_aabbs(aabb const *__restrict__ in, std::uint32_t const *__restrict__ ids,
                   aabb *__restrict__ out, std::uint64_t n) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = in[ids[i]];
}

template <class K> struct karras_delta {
    K const *codes;
    std::int64_t n;
    __device__ int operator()(std::int64_t i, std::int64_t j) const {
        if (j < 0 || j >= n)
            return -1;
        K const ci = codes[i];
        K const cj = codes[j];
        if (ci == cj) {
            std::uint64_t const diff = static_cast<std::uint64_t>(i) ^ static_cast<std::uint64_t>(j);
            if (diff == 0)
                return static_cast<int>(sizeof(K) * 8 + 64);
            return static_cast<int>(sizeof(K) * 8) + __clzll(static_cast<long long>(diff));
        }
        if constexpr (sizeof(K) == 4)
            return __clz(static_cast<int>(ci ^ cj));
        else
            return __clzll(static_cast<long long>(ci ^ cj));
    }
};

// Karras 2012 binary radix tree over sorted codes (one thread per internal node).
template <class K>
__global__ void __launch_bounds__(k_block)
    k_karras(K const *__restrict__ codes, std::int64_t n, binary_node *__restrict__ nodes,
             std::uint32_t *__restrict__ internal_parent, std::uint32_t *__restrict__ leaf_parent) {
    std::int64_t const i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n - 1)
        return;
    karras_delta<K> const delta{codes, n};
    int const dir = (delta(i, i + 1) - delta(i, i - 1) >= 0) ? 1 : -1;
    int const dmin = delta(i, i - dir);
    std::int64_t lmax = 2;
    while (delta(i, i + lmax * dir) > dmin)
        lmax <<= 1;
    std::int64_t l = 0;
    for (std::int64_t t = lmax >> 1; t > 0; t >>= 1)
        if (delta(i, i + (l + t) * dir) > dmin)
            l += t;
    std::int64_t const j = i + l * dir;
    std::int64_t const first = min(i, j);
    std::int64_t const last = max(i, j);
    int const dnode = delta(first, last);
    std::int64_t split = first;
    std::int64_t step = last - first;
    do {
        step = (step + 1) >> 1;
        std::int64_t const cand = split + step;
        if (cand < last && delta(first, cand) > dnode)
            split = cand;
    } while (step > 1);

    binary_node nd;
    nd.left_index = static_cast<std::uint32_t>(split);
    nd.left_kind = (split == first) ? k_kind_leaf : k_kind_internal;
    nd.right_index = static_cast<std::uint32_t>(split + 1);
    nd.right_kind = (split + 1 == last) ? k_kind_leaf : k_kind_internal;
    nodes[i] = nd;
    std::uint32_t const me2 = static_cast<std::uint32_t>(i) << 1;
    if (nd.left_kind == k_kind_internal)
        internal_parent[nd.left_index] = me2 | 0u;
    else
        leaf_parent[nd.left_index] = me2 | 0u;
    if (nd.right_kind == k_kind_internal)
        internal_parent[nd.right_index] = me2 | 1u;
    else
        leaf_parent[nd.right_index] = me2 | 1u;
}

// Bottom-up internal bounds: the second child to arrive at a node forms its union and climbs.
// Parent words hold (parent << 1) | slot.
__global__ void __launch_bounds__(k_block)
    k_binary_bounds(aabb const *__restrict__ leaf_aabbs, std::uint64_t n,
                    std::uint32_t const *__restrict__ leaf_parent,
                    std::uint32_t const *__restrict__ internal_parent, aabb *pending /* 2 per node */,
                    aabb *internal_bounds, unsigned int *arrivals, unsigned int *status) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    std::uint32_t pw = leaf_parent[i];
    aabb cur = leaf_aabbs[i];
    std::uint64_t guard = 0;
    while (pw != k_invalid_u32) {
        std::uint32_t const p = pw >> 1;
        std::uint32_t const slot = pw & 1u;
        if (p >= n - 1 || ++guard > n) {
            atomicOr(status, k_err_topology);
            return;
        }
        pending[2 * static_cast<std::uint64_t>(p) + slot] = cur;
        fence_acq_rel_gpu();
        if (atomicAdd(&arrivals[p], 1u) == 0u)
            return;
        fence_acq_rel_gpu();
        aabb l, r;
        {
            float const *pl = reinterpret_cast<float const *>(&pending[2 * static_cast<std::uint64_t>(p)]);
            float v[12];
#pragma unroll
            for (int k = 0; k < 12; ++k)
                v[k] = __ldcg(pl + k);
            l = aabb{v[0], v[1], v[2], v[3], v[4], v[5]};
            r = aabb{v[6], v[7], v[8], v[9], v[10], v[11]};
        }
        cur = aabb_union(l, r);
        internal_bounds[p] = cur;
        pw = internal_parent[p];
    }
}

// ---- level-synchronous collapse ------------------------------------------------------------------

struct collapse_item {
    std::uint32_t binary_index;
    std::uint32_t prefix_internal;
    std::uint32_t prefix_packed;
};

struct collapse_params {
    binary_node const *binary;
    aabb const *binary_bounds;
    aabb const *leaf_aabbs;
    std::uint64_t leaf_count;
    node4 *nodes;
    std::uint64_t node_capacity;
    collapse_item *lists[2];
    std::uint32_t *level_count; // [max_levels + 1]
    std::uint32_t *level_base;  // [max_levels + 1]
    std::uint32_t *tile_counter; // [max_levels]
    unsigned long long *tile_status; // tagged (level+1) << 34 | flag << 32 | value
    std::uint32_t *stack_bounds;     // [2]: internal, packed
    unsigned int *status;
    std::uint64_t list_capacity;     // items per level list (binary internal node count)
    long long wait_limit;            // polls before a look-back wait gives up (wait_limit())
};

constexpr unsigned long long k_ts_agg = 1ull << 32;
constexpr unsigned long long k_ts_incl = 2ull << 32;

// Decoupled look-back of one collapse tile: publishes the tile's aggregate, adds the published
// values of the tiles before it (tagged with this level, so a previous level's words never count)
// until an inclusive prefix is found, publishes the inclusive prefix and returns the exclusive
// one. A predecessor that stays unpublished for `limit` polls sets k_err_wait_timeout and ends the
// wait with the prefix gathered so far, so the launch always completes.
__device__ std::uint32_t collapse_tile_prefix(unsigned long long *st, std::uint32_t tile, unsigned long long tag,
                                              std::uint32_t block_total, unsigned int *status, long long limit) {
    std::uint32_t excl = 0;
    if (tile == 0) {
        atomicExch(&st[0], tag | k_ts_incl | block_total);
        return 0;
    }
    atomicExch(&st[tile], tag | k_ts_agg | block_total);
    long long spins = 0;
    std::int64_t j = static_cast<std::int64_t>(tile) - 1;
    while (j >= 0) {
        unsigned long long const s = *reinterpret_cast<volatile unsigned long long *>(&st[j]);
        if ((s & ~((1ull << 34) - 1)) != tag || (s & (3ull << 32)) == 0) {
            if (++spins > limit) {
                atomicOr(status, k_err_wait_timeout);
                break;
            }
            continue;
        }
        excl += static_cast<std::uint32_t>(s & 0xffffffffull);
        if ((s & (3ull << 32)) == k_ts_incl)
            break;
        --j;
    }
    atomicExch(&st[tile], tag | k_ts_incl | (excl + block_total));
    return excl;
}

// One level of the collapse: blocks claim tiles of k_block items from the level's counter in launch
// order (so a tile's look-back only ever waits on tiles claimed before it) until the level is
// exhausted.
__global__ void __launch_bounds__(k_block) k_collapse_level(collapse_params p, int level) {
    __shared__ std::uint32_t s_tile;
    __shared__ std::uint32_t s_prefix;
    __shared__ std::uint32_t s_scan[k_block / 32];
    std::uint32_t n_in = *reinterpret_cast<volatile std::uint32_t *>(&p.level_count[level]);
    if (n_in > p.list_capacity) {
        // only a broken binary hierarchy can hold more items on one level than internal nodes
        if (threadIdx.x == 0)
            atomicOr(p.status, k_err_collapse);
        n_in = 0;
    }
    std::uint32_t const base = *reinterpret_cast<volatile std::uint32_t *>(&p.level_base[level]);
    // selected, not indexed: a run-time index into the parameter array would copy it to local memory
    bool const odd = (level & 1) != 0;
    collapse_item const *items_in = odd ? p.lists[1] : p.lists[0];
    collapse_item *items_out = odd ? p.lists[0] : p.lists[1];
    unsigned const tid = threadIdx.x;
    unsigned const lane = tid & 31u;
    unsigned const warp = tid >> 5;
    unsigned long long const tag = static_cast<unsigned long long>(level + 1) << 34;

    for (;;) {
        if (tid == 0)
            s_tile = atomicAdd(&p.tile_counter[level], 1u);
        __syncthreads();
        std::uint32_t const tile = s_tile;
        __syncthreads();
        if (static_cast<std::uint64_t>(tile) * k_block >= n_in)
            break;
        std::uint32_t const i = tile * k_block + tid;
        bool const valid = i < n_in;

        std::uint32_t cidx[4] = {0, 0, 0, 0};
        std::uint32_t ckind[4] = {0, 0, 0, 0};
        int k = 0;
        std::uint32_t k_int = 0;
        collapse_item item{0, 0, 0};
        if (valid) {
            item = items_in[i];
            if (item.binary_index >= p.leaf_count - 1) {
                atomicOr(p.status, k_err_collapse);
            } else {
                binary_node const root = p.binary[item.binary_index];
                cidx[0] = root.left_index;
                ckind[0] = root.left_kind;
                cidx[1] = root.right_index;
                ckind[1] = root.right_kind;
                k = 2;
                // Expand the largest-area internal child (ties: smallest binary index) until four
                // children or only leaves remain; every index into cidx/ckind is a compile-time
                // constant, so both stay in registers.
#pragma unroll
                for (int step = 0; step < 2; ++step) {
                    int best = -1;
                    float best_area = -__int_as_float(0x7f800000);
                    std::uint32_t best_index = k_invalid_u32;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (c >= k || ckind[c] != k_kind_internal || cidx[c] >= p.leaf_count - 1)
                            continue;
                        float const area = aabb_half_area(p.binary_bounds[cidx[c]]);
                        if (best >= 0 && area < best_area)
                            continue;
                        if (best >= 0 && area == best_area && cidx[c] >= best_index)
                            continue;
                        best = c;
                        best_area = area;
                        best_index = cidx[c];
                    }
                    if (best < 0)
                        break;
                    binary_node const e = p.binary[best_index];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (c == best) {
                            cidx[c] = e.left_index;
                            ckind[c] = e.left_kind;
                        } else if (c == k) {
                            cidx[c] = e.right_index;
                            ckind[c] = e.right_kind;
                        }
                    }
                    ++k;
                }
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    k_int += (c < k && ckind[c] == k_kind_internal) ? 1u : 0u;
            }
        }

        // Block scan of internal-child counts.
        std::uint32_t incl = k_int;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            std::uint32_t const t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= static_cast<unsigned>(o))
                incl += t;
        }
        if (lane == 31)
            s_scan[warp] = incl;
        __syncthreads();
        std::uint32_t warp_prefix = 0, block_total = 0;
        for (int w = 0; w < k_block / 32; ++w) {
            if (static_cast<unsigned>(w) < warp)
                warp_prefix += s_scan[w];
            block_total += s_scan[w];
        }
        std::uint32_t const local_excl = warp_prefix + incl - k_int;

        // Decoupled look-back over tiles of this level.
        if (tid == 0)
            s_prefix = collapse_tile_prefix(p.tile_status, tile, tag, block_total, p.status, p.wait_limit);
        __syncthreads();
        std::uint32_t const tile_prefix = s_prefix;
        __syncthreads();

        if (valid && k > 0) {
            std::uint32_t const w = base + i;
            std::uint32_t const out_first = tile_prefix + local_excl;
            std::uint32_t const id_first = base + n_in + out_first;
            std::uint32_t const node_int = item.prefix_internal + (k_int > 0 ? k_int - 1u : 0u);
            std::uint32_t const node_pk = item.prefix_packed + static_cast<std::uint32_t>(k - 1);
            // only a broken binary hierarchy can produce more items than the list holds
            bool const room = static_cast<std::uint64_t>(out_first) + k_int <= p.list_capacity;
            if (!room)
                atomicOr(p.status, k_err_collapse);
            bool const node_ok = w < p.node_capacity;
            if (!node_ok)
                atomicOr(p.status, k_err_collapse);
            float4 *const dst = reinterpret_cast<float4 *>(p.nodes + (node_ok ? w : 0u));
            std::uint32_t m = 0;
            // Each child is written as two 16-byte stores straight from registers.
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                aabb bb{0, 0, 0, 0, 0, 0};
                std::uint64_t ref = 0;
                if (c < k) {
                    if (ckind[c] == k_kind_leaf) {
                        if (cidx[c] < p.leaf_count) {
                            bb = p.leaf_aabbs[cidx[c]];
                            ref = make_ref(cidx[c], 1u);
                        } else {
                            atomicOr(p.status, k_err_collapse);
                        }
                    } else {
                        if (cidx[c] < p.leaf_count - 1)
                            bb = p.binary_bounds[cidx[c]];
                        else
                            atomicOr(p.status, k_err_collapse);
                        ref = make_ref(id_first + m, 0u);
                        if (room)
                            items_out[out_first + m] = collapse_item{cidx[c], node_int, node_pk};
                        ++m;
                    }
                }
                if (node_ok) {
                    dst[2 * c] = make_float4(bb.min_x, bb.min_y, bb.min_z, bb.max_x);
                    dst[2 * c + 1] = make_float4(bb.max_y, bb.max_z, __uint_as_float(static_cast<std::uint32_t>(ref)),
                                                 __uint_as_float(static_cast<std::uint32_t>(ref >> 32)));
                }
            }
            atomicMax(&p.stack_bounds[0], node_int);
            atomicMax(&p.stack_bounds[1], node_pk);
        }
        if (valid && i == n_in - 1) {
            p.level_count[level + 1] = tile_prefix + local_excl + k_int;
            p.level_base[level + 1] = base + n_in;
        }
    }
}

// Starts the collapse at the binary root. The H-PLOC builder's cluster counter, when given, must
// read 2n - 1 (a complete hierarchy), else the collapse reports an error and produces no nodes.
__global__ void k_collapse_init(collapse_params p, std::uint32_t root_binary, std::uint32_t const *hploc_count,
                                std::uint32_t hploc_expected) {
    bool ok = true;
    if (hploc_count != nullptr && *hploc_count != hploc_expected) {
        atomicOr(p.status, k_err_hploc);
        ok = false;
    }
    p.lists[0][0] = collapse_item{root_binary, 0u, 0u};
    p.level_count[0] = ok ? 1u : 0u;
    p.level_base[0] = 0u;
}

// Sizes after `levels` levels: the node count is the base of the first empty level and the stack
// bounds the maxima the levels recorded; `pending` is set when level `levels` still holds items.
__global__ void k_collapse_summary(collapse_params p, int levels, collapse_summary *summary) {
    int l = 0;
    while (l < levels && p.level_count[l] != 0u)
        ++l;
    summary->node_count = p.level_base[l];
    summary->internal_bound = p.stack_bounds[0];
    summary->packed_bound = p.stack_bounds[1];
    summary->pending = p.level_count[l] != 0u ? 1u : 0u;
}

__global__ void __launch_bounds__(k_block)
    k_triangles(gwnb_geometry_f32 g, std::uint32_t const *__restrict__ ids, std::uint64_t n,
                triangle *__restrict__ tris, triangle48 *__restrict__ tri48, unsigned int *status) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    std::uint32_t const t = ids[i];
    if (t >= g.triangle_count) {
        atomicOr(status, k_err_index);
        return;
    }
    std::uint32_t const a = g.tri_i0[t], b = g.tri_i1[t], c = g.tri_i2[t];
    std::uint64_t const nv = g.vertex_count;
    if (a >= nv || b >= nv || c >= nv) {
        atomicOr(status, k_err_index);
        return;
    }
    float const ax = g.vertex_x[a], ay = g.vertex_y[a], az = g.vertex_z[a];
    float const e1x = __fsub_rn(g.vertex_x[b], ax), e1y = __fsub_rn(g.vertex_y[b], ay),
                e1z = __fsub_rn(g.vertex_z[b], az);
    float const e2x = __fsub_rn(g.vertex_x[c], ax), e2y = __fsub_rn(g.vertex_y[c], ay),
                e2z = __fsub_rn(g.vertex_z[c], az);
    tris[i] = triangle{ax, ay, az, e1x, e1y, e1z, e2x, e2y, e2z};
    if (tri48 != nullptr)
        tri48[i] = make_triangle48(ax, ay, az, e1x, e1y, e1z, e2x, e2y, e2z);
}

inline unsigned grid_for(std::uint64_t n, int block = k_block) {
    return static_cast<unsigned>((n + block - 1) / block);
}

} // namespace

// ---- host orchestration -----------------------------------------------------------------------

int build_scene_and_morton(gwnb_geometry_f32 const &g, int morton_bits, aabb *aabbs, void *codes,
                           cudaStream_t s) {
    std::uint64_t const nt = g.triangle_count;
    unsigned int *scene = nullptr;
    scratch_guard guard(s);
    guard.hold(scene);
    GWNB_TRY(alloc(&scene, 6, s));
    static unsigned int const init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    GWNB_CUDA_TRY(cudaMemcpyAsync(scene, init, sizeof(init), cudaMemcpyHostToDevice, s));
    unsigned const grid = static_cast<unsigned>(
        std::min<std::uint64_t>(grid_for(g.vertex_count), static_cast<std::uint64_t>(device_sm_count()) * 4));
    note_launch(), k_scene_bounds<<<std::max(1u, grid), k_block, 0, s>>>(g.vertex_x, g.vertex_y, g.vertex_z,
                                                          g.vertex_count, scene);
    if (morton_bits == 32)
        note_launch(), k_morton<std::uint32_t><<<grid_for(nt), k_block, 0, s>>>(
            g, scene, aabbs, static_cast<std::uint32_t *>(codes));
    else
        note_launch(), k_morton<std::uint64_t><<<grid_for(nt), k_block, 0, s>>>(
            g, scene, aabbs, static_cast<std::uint64_t *>(codes));
    GWNB_CUDA_TRY(cudaGetLastError());
    release(scene, s);
    return GWNB_OK;
}

// Preprocess: Morton codes, stable sort, gathered AABBs. Outputs are caller-owned.
int build_preprocess(gwnb_geometry_f32 const &g, int morton_bits, void *sorted_codes,
                     std::uint32_t *sorted_ids, aabb *sorted_aabbs, cudaStream_t s,
                     unsigned int *status) {
    std::uint64_t const nt = g.triangle_count;
    if (nt == 0)
        return GWNB_OK;
    int const kb = morton_bits / 8;
    aabb *aabbs = nullptr;
    unsigned char *codes = nullptr;
    scratch_guard guard(s);
    guard.hold(aabbs, codes);
    GWNB_TRY(alloc(&aabbs, nt, s));
    GWNB_TRY(alloc(&codes, nt * kb, s));
    GWNB_TRY(build_scene_and_morton(g, morton_bits, aabbs, codes, s));
    GWNB_TRY(radix_sort_pairs(codes, sorted_codes, nullptr, sorted_ids, nt, kb, morton_bits, s, status));
    note_launch(), k_gather_aabbs<<<grid_for(nt), k_block, 0, s>>>(aabbs, sorted_ids, sorted_aabbs, nt);
    GWNB_CUDA_TRY(cudaGetLastError());
    release(aabbs, s);
    release(codes, s);
    return GWNB_OK;
}

int build_binary_lbvh(void const *sorted_codes, int morton_bits, std::uint64_t n,
                      aabb const *sorted_aabbs, binary_node *nodes, std::uint32_t *internal_parent,
                      aabb *internal_bounds, cudaStream_t s, unsigned int *status) {
    if (n < 2)
        return GWNB_OK;
    std::uint64_t const ni = n - 1;
    std::uint32_t *leaf_parent = nullptr;
    aabb *pending = nullptr;
    unsigned int *arrivals = nullptr;
    scratch_guard guard(s);
    guard.hold(leaf_parent, pending, arrivals);
    GWNB_TRY(alloc(&leaf_parent, n, s));
    GWNB_TRY(alloc(&pending, 2 * ni, s));
    GWNB_TRY(alloc(&arrivals, ni, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(internal_parent, 0xff, ni * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(leaf_parent, 0xff, n * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(arrivals, 0, ni * sizeof(unsigned int), s));
    if (morton_bits == 32)
        note_launch(), k_karras<std::uint32_t><<<grid_for(ni), k_block, 0, s>>>(
            static_cast<std::uint32_t const *>(sorted_codes), static_cast<std::int64_t>(n), nodes,
            internal_parent, leaf_parent);
    else
        note_launch(), k_karras<std::uint64_t><<<grid_for(ni), k_block, 0, s>>>(
            static_cast<std::uint64_t const *>(sorted_codes), static_cast<std::int64_t>(n), nodes,
            internal_parent, leaf_parent);
    note_launch(), k_binary_bounds<<<grid_for(n), k_block, 0, s>>>(sorted_aabbs, n, leaf_parent, internal_parent,
                                                    pending, internal_bounds, arrivals, status);
    GWNB_CUDA_TRY(cudaGetLastError());
    release(leaf_parent, s);
    release(pending, s);
    release(arrivals, s);
    return GWNB_OK;
}

int build_binary_hploc(void const *sorted_codes, int morton_bits, std::uint64_t n,
                       aabb const *sorted_aabbs, std::uint32_t radius, binary_node *nodes,
                       std::uint32_t *internal_parent, aabb *internal_bounds, std::uint32_t *root,
                       cudaStream_t s, unsigned int *status, std::uint32_t *counter);

// Collapse a binary hierarchy into canonical breadth-first BVH4 nodes. With sync == false the first
// k_async_levels levels are enqueued without a host round trip and *summary (device memory) says
// whether the tree was deeper (summary->pending): the caller then repeats the collapse with sync ==
// true, which continues level batches until one comes back empty. The node count and both stack
// bounds land in *summary. hploc_count, when non-null, is the H-PLOC builder's cluster counter,
// checked on the device against 2n - 1.
int collapse_to_bvh4(binary_node const *binary, aabb const *binary_bounds, aabb const *leaf_aabbs,
                     std::uint64_t leaf_count, std::uint32_t root_binary, std::uint32_t const *hploc_count,
                     node4 *nodes, std::uint64_t node_capacity, collapse_summary *summary, bool sync,
                     cudaStream_t s, unsigned int *status) {
    constexpr int k_max_levels = 4096;
    constexpr int k_async_levels = 32;
    std::uint64_t const ni = leaf_count - 1;
    std::uint64_t const max_tiles = (ni + k_block - 1) / k_block;
    collapse_params p{};
    p.binary = binary;
    p.binary_bounds = binary_bounds;
    p.leaf_aabbs = leaf_aabbs;
    p.leaf_count = leaf_count;
    p.nodes = nodes;
    p.node_capacity = node_capacity;
    p.list_capacity = ni;
    p.wait_limit = wait_limit();
    std::uint32_t *words = nullptr;
    std::size_t const nwords = 3 * (k_max_levels + 1) + 2;
    scratch_guard guard(s);
    guard.hold(p.lists[0], p.lists[1], words, p.tile_status);
    GWNB_TRY(alloc(&p.lists[0], ni, s));
    GWNB_TRY(alloc(&p.lists[1], ni, s));
    GWNB_TRY(alloc(&words, nwords, s));
    GWNB_TRY(alloc(&p.tile_status, max_tiles, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(words, 0, nwords * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(p.tile_status, 0, max_tiles * sizeof(unsigned long long), s));
    p.level_count = words;
    p.level_base = words + (k_max_levels + 1);
    p.tile_counter = words + 2 * (k_max_levels + 1);
    p.stack_bounds = words + 3 * (k_max_levels + 1);
    p.status = status;
    note_launch(), k_collapse_init<<<1, 1, 0, s>>>(p, root_binary, hploc_count,
                                                   static_cast<std::uint32_t>(2 * leaf_count - 1));
    unsigned const grid = static_cast<unsigned>(
        std::min<std::uint64_t>(max_tiles, static_cast<std::uint64_t>(device_sm_count()) * 4));
    int level = 0;
    for (;;) {
        int const batch = sync && level > 0 ? 8 : k_async_levels;
        for (int b = 0; b < batch && level < k_max_levels; ++b, ++level)
            note_launch(), k_collapse_level<<<grid, k_block, 0, s>>>(p, level);
        GWNB_CUDA_TRY(cudaGetLastError());
        if (!sync)
            break;
        std::uint32_t c = 0;
        GWNB_CUDA_TRY(cudaMemcpyAsync(&c, p.level_count + level, sizeof(c), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
        if (c == 0)
            break;
        if (level >= k_max_levels)
            return set_error(GWNB_INTERNAL_ERROR, "bvh.build.collapse: tree deeper than 4096 levels.");
    }
    note_launch(), k_collapse_summary<<<1, 1, 0, s>>>(p, level, summary);
    GWNB_CUDA_TRY(cudaGetLastError());
    release(p.lists[0], s);
    release(p.lists[1], s);
    release(words, s);
    release(p.tile_status, s);
    return GWNB_OK;
}

namespace {
// Tile 1 of a level waits on tile 0, which nothing publishes.
__global__ void k_collapse_wait_probe(unsigned long long *st, unsigned int *status, long long limit) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
        (void)collapse_tile_prefix(st, 1u, 1ull << 34, 1u, status, limit);
}
} // namespace

// The collapse's look-back wait on a predecessor tile that is never published: one thread runs the
// wait of tile 1 against a zeroed tile-status array; it gives up after wait_limit() polls and sets
// k_err_wait_timeout in *status.
int collapse_wait_probe(unsigned int *status, cudaStream_t s) {
    unsigned long long *st = nullptr;
    GWNB_TRY(alloc(&st, 2, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(st, 0, 2 * sizeof(unsigned long long), s));
    note_launch(), k_collapse_wait_probe<<<1, 32, 0, s>>>(st, status, wait_limit());
    cudaError_t const e = cudaGetLastError();
    release(st, s);
    if (e != cudaSuccess)
        return set_cuda_error(e, "collapse wait probe");
    return GWNB_OK;
}

int build_triangles(gwnb_geometry_f32 const &g, std::uint32_t const *ids, std::uint64_t n,
                    triangle *tris, triangle48 *tri48, cudaStream_t s, unsigned int *status) {
    if (n == 0)
        return GWNB_OK;
    note_launch(), k_triangles<<<grid_for(n), k_block, 0, s>>>(g, ids, n, tris, tri48, status);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

} // namespace gwnb
