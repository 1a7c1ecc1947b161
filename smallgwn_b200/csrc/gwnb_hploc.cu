// H-PLOC binary builder (Benthin, Meister, Barczak, Mehalwal, Tsakok, Kensler: "H-PLOC:
// Hierarchical Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy Construction",
// HPG 2024).
//
// Every decision that shapes the topology follows smallgwn's builder
// (detail/gwn_bvh_build_hploc.cuh:104-478), so the two produce the same binary tree up to the
// numbering of internal nodes:
//   - Morton boundaries with the index extension of equal codes (:139-151) and the parent choice
//     between the left and right boundary (:152-158);
//   - half-warp cluster lists: a range is merged only when it spans more than 16 leaves, down to
//     16 clusters (1 for the root range) (:446-477, :425-436);
//   - nearest neighbour within radius r <= 8 by half-area of the union, ranked by a packed 32-bit
//     key (area bits << 1 with the low 4 bits replaced by (offset - 1) << 1 | direction parity)
//     so ties break identically at both endpoints (:195-241);
//   - mutual nearest neighbours merge, the lower lane keeps the merged cluster, survivors compact
//     to the low lanes (:300-399).
// Internal ids are allocated per warp iteration from a global counter, so their numbering (not
// the tree) depends on scheduling, as in smallgwn.
#include "gwnb_internal.cuh"

namespace gwnb {

namespace {

constexpr int k_hploc_block = 128;
constexpr std::uint32_t k_threshold = 16u;
constexpr std::uint32_t k_max_radius = 8u;
constexpr std::uint32_t k_inv = 0xffffffffu;

__device__ inline aabb shfl_aabb(aabb const &v, int src) {
    return aabb{__shfl_sync(0xffffffffu, v.min_x, src), __shfl_sync(0xffffffffu, v.min_y, src),
                __shfl_sync(0xffffffffu, v.min_z, src), __shfl_sync(0xffffffffu, v.max_x, src),
                __shfl_sync(0xffffffffu, v.max_y, src), __shfl_sync(0xffffffffu, v.max_z, src)};
}

template <class K> struct hploc_delta {
    K const *codes;
    __device__ std::uint64_t operator()(std::uint32_t a, std::uint32_t b) const {
        K const ka = codes[a];
        K const kb = codes[b];
        if constexpr (sizeof(K) == 4) {
            std::uint64_t const ca = (static_cast<std::uint64_t>(ka) << 32) | a;
            std::uint64_t const cb = (static_cast<std::uint64_t>(kb) << 32) | b;
            return ca ^ cb;
        } else {
            std::uint64_t const d = static_cast<std::uint64_t>(ka ^ kb);
            return d == 0 ? static_cast<std::uint64_t>(a ^ b) : d;
        }
    }
};

struct hploc_params {
    std::uint32_t n;
    std::uint32_t radius;
    aabb const *leaf_aabbs;
    binary_node *nodes;
    aabb *internal_bounds;
    std::uint32_t *internal_parent; // (parent << 1) | slot
    std::uint32_t *cluster_indices;
    std::uint32_t *boundary_parent;
    std::uint32_t *cluster_count;
    unsigned int *status;
};

template <class K> __global__ void __launch_bounds__(k_hploc_block) k_hploc(hploc_params p, K const *codes) {
    unsigned const lane = threadIdx.x & 31u;
    std::uint32_t const n = p.n;
    std::uint64_t const gidx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    hploc_delta<K> const delta{codes};

    auto parent_is_right = [&](std::uint32_t left, std::uint32_t right) {
        return left == 0 || (right != n - 1 && delta(right, right + 1) < delta(left - 1, left));
    };
    auto cluster_bounds_of = [&](std::uint32_t c) -> aabb {
        if (c < n)
            return p.leaf_aabbs[c];
        if (c >= 2 * n - 1) {
            atomicOr(p.status, k_err_hploc);
            return aabb{0, 0, 0, 0, 0, 0};
        }
        float const *src = reinterpret_cast<float const *>(&p.internal_bounds[c - n]);
        return aabb{__ldcg(src), __ldcg(src + 1), __ldcg(src + 2), __ldcg(src + 3), __ldcg(src + 4),
                    __ldcg(src + 5)};
    };
    auto load_list = [&](std::uint32_t start, std::uint32_t end, std::uint32_t &cid,
                         std::uint32_t offset) -> std::uint32_t {
        std::uint32_t const idx = lane - offset; // wraps for lanes below offset
        std::uint32_t const cnt = min(end - start, k_threshold);
        bool const valid = idx < cnt;
        if (valid)
            cid = __ldcg(&p.cluster_indices[start + idx]);
        return __popc(__ballot_sync(0xffffffffu, valid && cid != k_inv));
    };

    auto nearest = [&](std::uint32_t num, aabb const &mine) -> std::uint32_t {
        constexpr std::uint32_t k_nmask = (1u << 4) - 1u;
        std::uint32_t best = 0xffffffffu;
#pragma unroll
        for (std::uint32_t r = 1; r <= k_max_radius; ++r) {
            if (r > p.radius)
                break;
            std::uint32_t const nl = lane + r;
            bool const nvalid = nl < num;
            int const safe_n = nvalid ? static_cast<int>(nl) : static_cast<int>(lane);
            aabb const other = shfl_aabb(mine, safe_n);
            std::uint32_t right_key = 0xffffffffu;
            if (nvalid) {
                float const area = aabb_half_area(aabb_union(mine, other));
                std::uint32_t const akey = (__float_as_uint(area) << 1) & ~k_nmask;
                std::uint32_t const rel = (r - 1u) << 1;
                right_key = akey | rel | ((nl & 1u) ^ 1u);
                best = min(best, akey | rel | (lane & 1u));
            }
            std::uint32_t nk = __shfl_sync(0xffffffffu, best, safe_n);
            if (nvalid)
                nk = min(nk, right_key);
            int const ll = static_cast<int>(lane) - static_cast<int>(r);
            std::uint32_t const shifted = __shfl_sync(0xffffffffu, nk, ll >= 0 ? ll : static_cast<int>(lane));
            if (ll >= 0)
                best = shifted;
        }
        std::uint32_t const off = ((best & k_nmask) >> 1) + 1u;
        bool const right = ((best ^ lane) & 1u) == 0u;
        return right ? lane + off : lane - off;
    };

    auto merge = [&](std::uint32_t num, std::uint32_t nn, std::uint32_t &cid, aabb &b) -> std::uint32_t {
        bool const active = lane < num;
        bool const nvalid = nn < num && nn != lane;
        if (active && !nvalid)
            atomicOr(p.status, k_err_hploc);
        std::uint32_t const safe = nvalid ? nn : lane;
        std::uint32_t const nn_of_nn = __shfl_sync(0xffffffffu, safe, static_cast<int>(safe));
        bool const mutual = active && nvalid && lane == nn_of_nn;
        bool const do_merge = mutual && lane < safe;
        unsigned const mmask = __ballot_sync(0xffffffffu, do_merge);
        std::uint32_t const mcount = __popc(mmask);
        std::uint32_t base = 0;
        if (lane == 0 && mcount > 0)
            base = atomicAdd(p.cluster_count, mcount);
        base = __shfl_sync(0xffffffffu, base, 0);
        std::uint32_t const rel = __popc(mmask & ((1u << lane) - 1u));
        std::uint32_t const ncid = __shfl_sync(0xffffffffu, cid, static_cast<int>(safe));
        aabb const nb = shfl_aabb(b, static_cast<int>(safe));
        if (do_merge) {
            std::uint32_t const merged = base + rel;
            if (merged < n || merged >= 2 * n - 1) {
                atomicOr(p.status, k_err_hploc);
            } else {
                aabb const mb = aabb_union(b, nb);
                std::uint32_t const iid = merged - n;
                binary_node nd;
                nd.left_index = cid < n ? cid : cid - n;
                nd.left_kind = cid < n ? k_kind_leaf : k_kind_internal;
                nd.right_index = ncid < n ? ncid : ncid - n;
                nd.right_kind = ncid < n ? k_kind_leaf : k_kind_internal;
                p.nodes[iid] = nd;
                p.internal_bounds[iid] = mb;
                if (nd.left_kind == k_kind_internal)
                    p.internal_parent[nd.left_index] = (iid << 1) | 0u;
                if (nd.right_kind == k_kind_internal)
                    p.internal_parent[nd.right_index] = (iid << 1) | 1u;
                cid = merged;
                b = mb;
            }
        }
        unsigned const keep = __ballot_sync(0xffffffffu, do_merge || !mutual);
        int const src = __fns(keep, 0u, static_cast<int>(lane) + 1);
        int const safe_src = src == -1 ? static_cast<int>(lane) : src;
        std::uint32_t const scid = __shfl_sync(0xffffffffu, cid, safe_src);
        aabb const sb = shfl_aabb(b, safe_src);
        if (src == -1) {
            cid = k_inv;
        } else {
            cid = scid;
            b = sb;
        }
        return num - mcount;
    };

    auto ploc = [&](int sel, std::uint32_t left, std::uint32_t right, std::uint32_t split, bool fin) {
        std::uint32_t const l = __shfl_sync(0xffffffffu, left, sel);
        std::uint32_t const r_end = __shfl_sync(0xffffffffu, right, sel) + 1u;
        std::uint32_t const s = __shfl_sync(0xffffffffu, split, sel);
        std::uint32_t cid = k_inv;
        std::uint32_t const nl = load_list(l, s, cid, 0u);
        std::uint32_t const nr = load_list(s, r_end, cid, nl);
        std::uint32_t num = nl + nr;
        aabb b{0, 0, 0, 0, 0, 0};
        if (lane < num)
            b = cluster_bounds_of(cid);
        std::uint32_t const threshold = __shfl_sync(0xffffffffu, fin ? 1u : k_threshold, sel);
        int guard = 0;
        while (num > threshold) {
            std::uint32_t const prev = num;
            std::uint32_t const nn = nearest(num, b);
            num = merge(num, nn, cid, b);
            if (num == prev || ++guard > 64) {
                atomicOr(p.status, k_err_hploc);
                break;
            }
        }
        if (lane < nl + nr)
            p.cluster_indices[l + lane] = cid;
    };

    std::uint32_t left = static_cast<std::uint32_t>(gidx < n ? gidx : 0);
    std::uint32_t right = left;
    std::uint32_t split = 0;
    bool active = gidx < n;
    int outer_guard = 0;
    while (__ballot_sync(0xffffffffu, active) != 0u) {
        if (active) {
            std::uint32_t prev = k_inv;
            if (parent_is_right(left, right)) {
                prev = atomicExch(&p.boundary_parent[right], left);
                if (prev != k_inv) {
                    fence_acq_rel_gpu();
                    split = right + 1;
                    right = prev;
                }
            } else {
                prev = atomicExch(&p.boundary_parent[left - 1], right);
                if (prev != k_inv) {
                    fence_acq_rel_gpu();
                    split = left;
                    left = prev;
                }
            }
            if (prev == k_inv)
                active = false;
        }
        // a lane that acquired its sibling's range above orders the whole warp's reads of it
        __syncwarp();
        std::uint32_t const size = right - left + 1u;
        bool const fin = active && size == n;
        unsigned mask = __ballot_sync(0xffffffffu, (active && size > k_threshold) || fin);
        bool const merged_any = mask != 0u;
        while (mask != 0u) {
            int const sel = __ffs(static_cast<int>(mask)) - 1;
            ploc(sel, left, right, split, fin);
            mask &= mask - 1u;
        }
        // one release for every range this warp rewrote, before its next boundary exchange: the
        // lanes that wrote a range's list are ordered before its owner lane by the warp barrier
        __syncwarp();
        if (merged_any)
            fence_acq_rel_gpu();
        if (++outer_guard > 4096) {
            atomicOr(p.status, k_err_hploc);
            break;
        }
    }
}

__global__ void k_iota(std::uint32_t *v, std::uint32_t n) {
    std::uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = i;
}

} // namespace

// H-PLOC over n sorted leaves. The cluster counter ends at 2n - 1 when the hierarchy is complete,
// and the root is then internal node n - 2. With a caller-owned `counter` (one device word that
// must outlive the check) the call only enqueues work and the caller checks the counter on the
// device; with counter == nullptr it synchronizes the stream and checks it on the host.
int build_binary_hploc(void const *sorted_codes, int morton_bits, std::uint64_t n,
                       aabb const *sorted_aabbs, std::uint32_t radius, binary_node *nodes,
                       std::uint32_t *internal_parent, aabb *internal_bounds, std::uint32_t *root,
                       cudaStream_t s, unsigned int *status, std::uint32_t *counter) {
    *root = k_invalid_u32;
    if (n < 2)
        return GWNB_OK;
    if (n > 0x7fffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.binary.hploc: too many primitives.");
    bool const deferred_check = counter != nullptr;
    std::uint32_t *cluster = nullptr, *boundary = nullptr, *own_counter = nullptr;
    scratch_guard guard(s);
    guard.hold(cluster, boundary, own_counter);
    GWNB_TRY(alloc(&cluster, n, s));
    GWNB_TRY(alloc(&boundary, n, s));
    if (!deferred_check) {
        GWNB_TRY(alloc(&own_counter, 1, s));
        counter = own_counter;
    }
    GWNB_CUDA_TRY(cudaMemsetAsync(boundary, 0xff, n * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(internal_parent, 0xff, (n - 1) * sizeof(std::uint32_t), s));
    std::uint32_t const n32 = static_cast<std::uint32_t>(n);
    GWNB_CUDA_TRY(cudaMemcpyAsync(counter, &n32, sizeof(n32), cudaMemcpyHostToDevice, s));
    note_launch(), k_iota<<<(n32 + 255) / 256, 256, 0, s>>>(cluster, n32);
    hploc_params p{n32, radius, sorted_aabbs, nodes, internal_bounds, internal_parent, cluster,
                   boundary, counter, status};
    unsigned const grid = static_cast<unsigned>((n + k_hploc_block - 1) / k_hploc_block);
    if (morton_bits == 32)
        note_launch(), k_hploc<std::uint32_t><<<grid, k_hploc_block, 0, s>>>(p, static_cast<std::uint32_t const *>(sorted_codes));
    else
        note_launch(), k_hploc<std::uint64_t><<<grid, k_hploc_block, 0, s>>>(p, static_cast<std::uint64_t const *>(sorted_codes));
    GWNB_CUDA_TRY(cudaGetLastError());
    if (deferred_check) {
        release(cluster, s);
        release(boundary, s);
        *root = n32 - 2;
        return GWNB_OK;
    }
    std::uint32_t host_count = 0;
    unsigned int host_status = 0;
    GWNB_CUDA_TRY(cudaMemcpyAsync(&host_count, counter, sizeof(host_count), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(&host_status, status, sizeof(host_status), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    release(cluster, s);
    release(boundary, s);
    release(own_counter, s);
    if ((host_status & k_err_hploc) != 0u || host_count != 2 * n32 - 1)
        return set_error(GWNB_INTERNAL_ERROR,
                         "bvh.build.binary.hploc: H-PLOC builder did not converge to a complete binary hierarchy.");
    *root = n32 - 2;
    return GWNB_OK;
}

} // namespace gwnb
