// Adjoint of the Taylor winding-number batch (orders 0 and 1): the vector-Jacobian product of
// L = sum_q g_q w(q) with respect to the mesh's vertex positions and the query points. smallgwn has
// no such entry point; its query gradient (gwn_compute_winding_gradient_taylor_batch,
// include/gwn/gwn_query.cuh:688-756) is the dL/dq half of it for g = 1.
//
// w(q) = (1/4pi) [ sum over accepted child slots s of F_s(q - P_s; N_s, M_s)
//                + sum over the triangles t reached in the near field of Omega_t(q) ],
// with the slot moments of the moment refit: N = sum n_t, P = sum A_t c_t / sum A_t and
// M_ij = sum n_t,i c_t,j - N_i P_j (n_t = (e1 x e2)/2, A_t = |n_t|, c_t the centroid). The acceptance
// decisions are piecewise constant and carry no derivative. The backward pass recomputes the
// traversal instead of storing it:
//   1. k_adjoint_traverse: the forward's warp-cooperative traversal (same decisions). Every
//      accepted slot receives dL/dN_s, dL/dP_s and (order 1) dL/dM_s, summed over the lanes of a
//      warp before one atomic add per value; every near-field triangle receives dL/dv0,v1,v2; every
//      query receives dL/dq.
//   2. k_adjoint_triangles: per triangle, a walk over the slots that contain it (its leaf slot,
//      then the parent slots up to the root) applies the chain rule through N, M and P:
//        dL/dn_t += dL/dN_s + G_s (c_t - P_s),  dL/dc_t += G_s n_t + (A_t / A_s) H_s,
//        dL/dA_t += H_s . (c_t - P_s) / A_s,     H_s = dL/dP_s - G_s N_s,
//      with G_s = dL/dM_s (symmetric), then through n_t, A_t = |n_t| and c_t to the vertices, and
//      adds the near-field terms; vertex gradients are scattered with atomics.
// Slots of zero area (P at the box centre) pass no gradient through P.
#include "gwnb_field.cuh"

#include <algorithm>

namespace gwnb {

int query_order(aabb const *root_bounds, float const *qx, float const *qy, float const *qz, std::uint64_t n,
                std::uint32_t *order, cudaStream_t s, unsigned int *status);

namespace {

using namespace field;

// Per child slot: dL/dN (3), dL/dP (3), then for order 1 dL/dM over xx yy zz xy yz zx (6).
template <int Order> struct slot_floats {
    static constexpr int value = Order == 0 ? 6 : 12;
};

struct adjoint_params {
    float4 const *qnodes;
    std::uint32_t const *qcounts;
    triangle48 const *tri48;
    std::uint64_t primitive_count;
    std::uint64_t node_count;
    std::uint64_t root_ref;
    float const *qx;
    float const *qy;
    float const *qz;
    std::uint32_t const *order; // sorted position -> query index (nullptr: identity)
    float const *grad_out;
    float *dqx;
    float *dqy;
    float *dqz;
    float *slot_grad; // node_count * 4 * slot_floats (nullptr: no vertex gradients)
    float *tri_grad;  // primitive_count * 9 (nullptr: no vertex gradients)
    std::uint64_t n;
    float beta2;
    unsigned int *status;
};

// Adds the shares of the lanes in `mask` (warp-uniform; other lanes hold zeros) to dst[0..K),
// K <= 16. A lone lane adds its own share. Otherwise a recursive-halving reduce-scatter: at stride
// d = 1, 2, 4, 8 every lane keeps half of its remaining values (the lower half when its bit d is
// clear) and adds its partner's copy of that half, so after four steps lane l holds the sum over its
// 16-lane group of value bitrev4(l); one more exchange across the two groups completes the sums
// (16 shuffles where a butterfly per value would take 5 K), and 16 lanes add the K totals with one
// coalesced atomic instruction. Every lane of the warp must call it.
template <int K>
__device__ __forceinline__ void warp_scatter_add(float *dst, float const (&v)[K], unsigned mask, unsigned lane) {
    static_assert(K <= 16, "reduce-scatter holds at most 16 values");
    if (__popc(mask) == 1) {
        if (((mask >> lane) & 1u) != 0u) {
#pragma unroll
            for (int k = 0; k < K; ++k)
                atomicAdd(dst + k, v[k]);
        }
        return;
    }
    float r[16];
#pragma unroll
    for (int k = 0; k < 16; ++k)
        r[k] = k < K ? v[k] : 0.0f;
#pragma unroll
    for (int d = 1, m = 16; d <= 8; d <<= 1, m >>= 1) {
        bool const upper = (lane & static_cast<unsigned>(d)) != 0u;
#pragma unroll
        for (int j = 0; j < m / 2; ++j) {
            float const send = upper ? r[j] : r[j + m / 2];
            float const keep = upper ? r[j + m / 2] : r[j];
            r[j] = keep + __shfl_xor_sync(0xffffffffu, send, d);
        }
    }
    r[0] += __shfl_xor_sync(0xffffffffu, r[0], 16);
    unsigned const idx = __brev(lane & 15u) >> 28;
    if (lane < 16u && idx < static_cast<unsigned>(K))
        atomicAdd(dst + idx, r[0]);
}

template <int Order, int Cap>
__global__ void __launch_bounds__(256, 4) k_adjoint_traverse(adjoint_params p) {
    static_assert(Cap <= 64, "warp stack holds at most 64 entries");
    constexpr int Q = qnode_traits<Order>::k_f4_per_child;
    constexpr int SF = slot_floats<Order>::value;
    unsigned const lane = threadIdx.x & 31u;
    std::uint64_t const idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool const valid = idx < p.n;
    unsigned const full = __ballot_sync(0xffffffffu, valid);
    if (full == 0u)
        return;
    std::uint32_t const qi = valid ? (p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx)) : 0u;
    float const qx = valid ? p.qx[qi] : 0.0f;
    float const qy = valid ? p.qy[qi] : 0.0f;
    float const qz = valid ? p.qz[qi] : 0.0f;
    float const gam = valid ? p.grad_out[qi] * (1.0f / (4.0f * k_pi_f)) : 0.0f;
    bool const want_slots = p.slot_grad != nullptr;
    float dqx = 0.0f, dqy = 0.0f, dqz = 0.0f;

    // near field of triangles [first, first + cnt) for the lanes in `take` (all lanes call)
    auto leaf = [&](std::uint32_t first, std::uint32_t cnt, bool take, unsigned tmask) {
        for (std::uint32_t k = 0; k < cnt; ++k) {
            std::uint64_t const t = static_cast<std::uint64_t>(first) + k;
            if (t >= p.primitive_count)
                break;
            float v[9];
#pragma unroll
            for (int j = 0; j < 9; ++j)
                v[j] = 0.0f;
            if (take) {
                float4 const A = __ldg(&p.tri48[t].a);
                float4 const B = __ldg(&p.tri48[t].b);
                float4 const C = __ldg(&p.tri48[t].c);
                vertex_grad const vg =
                    solid_angle_vertex_grad(A.x - qx, A.y - qy, A.z - qz, A.w, B.x, B.y, B.z, B.w, C.x);
                v[0] = gam * vg.a.x;
                v[1] = gam * vg.a.y;
                v[2] = gam * vg.a.z;
                v[3] = gam * vg.b.x;
                v[4] = gam * vg.b.y;
                v[5] = gam * vg.b.z;
                v[6] = gam * vg.c.x;
                v[7] = gam * vg.c.y;
                v[8] = gam * vg.c.z;
                dqx -= v[0] + v[3] + v[6];
                dqy -= v[1] + v[4] + v[7];
                dqz -= v[2] + v[5] + v[8];
            }
            if (want_slots)
                warp_scatter_add<9>(p.tri_grad + t * 9, v, tmask, lane);
        }
    };

    bool overflow = false;
    if (ref_leaf(p.root_ref)) {
        leaf(static_cast<std::uint32_t>(ref_offset(p.root_ref)), ref_count(p.root_ref), valid, full);
    } else {
        std::uint32_t node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
        unsigned mask = full;
        std::uint32_t st_node0 = 0, st_node1 = 0;
        unsigned st_mask0 = 0, st_mask1 = 0;
        int sp = 0;
        for (;;) {
            if (node >= p.node_count)
                break;
            bool const active = ((mask >> lane) & 1u) != 0u;
            float4 const *nd = p.qnodes + static_cast<std::uint64_t>(node) * (4 * Q);
            std::uint32_t next = k_invalid_u32;
            unsigned next_mask = 0u;
#pragma unroll 1
            for (int s = 0; s < 4; ++s) {
                float4 const a = __ldg(nd + s * Q);
                if (a.w < 0.0f)
                    continue;
                float4 const b = __ldg(nd + s * Q + 1);
                bool desc = false, acc = false;
                float sv[SF];
#pragma unroll
                for (int j = 0; j < SF; ++j)
                    sv[j] = 0.0f;
                if (active) {
                    float const rx = qx - a.x, ry = qy - a.y, rz = qz - a.z;
                    float const q2 = accept_dist2(rx, ry, rz);
                    desc = !far_accepted(q2, a.w, p.beta2);
                    if (!desc) {
                        float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
                        float const w = far_field<Order, true>(rx, ry, rz, q2, b, nd + s * Q + 2, g0, g1, g2);
                        if (isfinite(w)) {
                            acc = true;
                            dqx += gam * g0;
                            dqy += gam * g1;
                            dqz += gam * g2;
                            float const m1 = rsqrtf(q2);
                            float const m2 = m1 * m1;
                            float const nx = rx * m1, ny = ry * m1, nz = rz * m1;
                            // dF/dN = -r^ / |r|^2; dF/dP = -dF/dq
                            sv[0] = -gam * m2 * nx;
                            sv[1] = -gam * m2 * ny;
                            sv[2] = -gam * m2 * nz;
                            sv[3] = -gam * g0;
                            sv[4] = -gam * g1;
                            sv[5] = -gam * g2;
                            if constexpr (Order >= 1) {
                                // dF/dM_ij = (delta_ij - 3 r^_i r^_j) / |r|^3
                                float const k = gam * m2 * m1;
                                sv[6] = k * (1.0f - 3.0f * nx * nx);
                                sv[7] = k * (1.0f - 3.0f * ny * ny);
                                sv[8] = k * (1.0f - 3.0f * nz * nz);
                                sv[9] = -3.0f * k * nx * ny;
                                sv[10] = -3.0f * k * ny * nz;
                                sv[11] = -3.0f * k * nz * nx;
                            }
                        } else {
                            desc = true;
                        }
                    }
                }
                if (want_slots) {
                    unsigned const amask = __ballot_sync(0xffffffffu, acc);
                    if (amask != 0u)
                        warp_scatter_add<SF>(p.slot_grad + (static_cast<std::uint64_t>(node) * 4 + s) * SF, sv,
                                             amask, lane);
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
                    std::uint32_t const cnt =
                        (ref & k_qref_multi) ? p.qcounts[static_cast<std::uint64_t>(node) * 4 + s] : 1u;
                    leaf(ref & k_qref_index_mask, cnt, desc, dmask);
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
    if (!valid)
        return;
    if (overflow) {
        atomicOr(p.status, k_err_stack_overflow);
        dqx = dqy = dqz = __int_as_float(0x7fc00000);
    }
    if (p.dqx != nullptr) {
        p.dqx[qi] = dqx;
        p.dqy[qi] = dqy;
        p.dqz[qi] = dqz;
    }
}

// Leaf slot of every sorted triangle: (node << 2) | slot.
__global__ void __launch_bounds__(256)
    k_leaf_slots(node4 const *__restrict__ nodes, std::uint64_t node_count, std::uint64_t primitive_count,
                 std::uint32_t *__restrict__ tri_slot) {
    std::uint64_t const n = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= node_count)
        return;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        std::uint64_t const r = nodes[n].c[s].reference;
        if (!ref_leaf(r))
            continue;
        std::uint64_t const first = ref_offset(r);
        std::uint32_t const cnt = ref_count(r);
        for (std::uint32_t k = 0; k < cnt; ++k)
            if (first + k < primitive_count)
                tri_slot[first + k] = static_cast<std::uint32_t>(n * 4 + s);
    }
}

struct adjoint_tri_params {
    float4 const *qnodes;
    std::uint32_t const *qcounts;
    triangle const *triangles;
    std::uint64_t primitive_count;
    std::uint64_t node_count;
    std::uint32_t const *tri_slot;
    std::uint32_t const *parent_slot;
    float const *payload;         // per-node moment payload; area is its first float
    std::uint64_t payload_floats; // floats per node payload
    float const *slot_grad;
    float const *tri_grad;
    std::uint32_t const *primitive_indices;
    gwnb_geometry_f32 g;
    float *dvx;
    float *dvy;
    float *dvz;
    unsigned int *status;
};

// Area-weighted normal, centroid and area of a record, formed as the moment refit forms them.
struct tri_terms {
    float nx, ny, nz, cx, cy, cz, area, e1x, e1y, e1z, e2x, e2y, e2z;
};

__device__ __forceinline__ tri_terms triangle_terms(triangle const &t) {
    tri_terms r;
    float const ax = t.v0_x, ay = t.v0_y, az = t.v0_z;
    float const bx = ax + t.e1_x, by = ay + t.e1_y, bz = az + t.e1_z;
    float const cx = ax + t.e2_x, cy = ay + t.e2_y, cz = az + t.e2_z;
    r.cx = (ax + bx + cx) / 3.0f;
    r.cy = (ay + by + cy) / 3.0f;
    r.cz = (az + bz + cz) / 3.0f;
    r.e1x = bx - ax;
    r.e1y = by - ay;
    r.e1z = bz - az;
    r.e2x = cx - ax;
    r.e2y = cy - ay;
    r.e2z = cz - az;
    r.nx = 0.5f * (r.e1y * r.e2z - r.e1z * r.e2y);
    r.ny = 0.5f * (r.e1z * r.e2x - r.e1x * r.e2z);
    r.nz = 0.5f * (r.e1x * r.e2y - r.e1y * r.e2x);
    r.area = sqrtf(rmax(r.nx * r.nx + r.ny * r.ny + r.nz * r.nz, 0.0f));
    return r;
}

template <int Order>
__global__ void __launch_bounds__(256) k_adjoint_triangles(adjoint_tri_params p) {
    constexpr int Q = qnode_traits<Order>::k_f4_per_child;
    constexpr int SF = slot_floats<Order>::value;
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= p.primitive_count)
        return;
    tri_terms const tt = triangle_terms(p.triangles[t]);
    float dnx = 0.0f, dny = 0.0f, dnz = 0.0f, dcx = 0.0f, dcy = 0.0f, dcz = 0.0f, dA = 0.0f;
    std::uint32_t slot = p.tri_slot != nullptr ? p.tri_slot[t] : k_invalid_u32;
    std::uint64_t guard = 0;
    while (slot != k_invalid_u32) {
        std::uint64_t const node = slot >> 2;
        int const s = static_cast<int>(slot & 3u);
        if (node >= p.node_count || ++guard > p.node_count + 1) {
            atomicOr(p.status, k_err_topology);
            break;
        }
        float4 const *sc = p.qnodes + (node * 4 + s) * Q;
        float4 const a = __ldg(sc);     // P, r2
        float4 const b = __ldg(sc + 1); // N, ref
        float const *G = p.slot_grad + (node * 4 + s) * SF;
        float const dx = tt.cx - a.x, dy = tt.cy - a.y, dz = tt.cz - a.z;
        dnx += G[0];
        dny += G[1];
        dnz += G[2];
        float hx = G[3], hy = G[4], hz = G[5];
        if constexpr (Order >= 1) {
            float const gxx = G[6], gyy = G[7], gzz = G[8], gxy = G[9], gyz = G[10], gzx = G[11];
            dnx += gxx * dx + gxy * dy + gzx * dz;
            dny += gxy * dx + gyy * dy + gyz * dz;
            dnz += gzx * dx + gyz * dy + gzz * dz;
            dcx += gxx * tt.nx + gxy * tt.ny + gzx * tt.nz;
            dcy += gxy * tt.nx + gyy * tt.ny + gyz * tt.nz;
            dcz += gzx * tt.nx + gyz * tt.ny + gzz * tt.nz;
            hx -= gxx * b.x + gxy * b.y + gzx * b.z;
            hy -= gxy * b.x + gyy * b.y + gyz * b.z;
            hz -= gzx * b.x + gyz * b.y + gzz * b.z;
        }
        // total area of the slot
        std::uint32_t const ref = __float_as_uint(b.w);
        float area_s;
        if ((ref & k_qref_leaf) != 0u) {
            std::uint32_t const cnt = (ref & k_qref_multi) ? p.qcounts[node * 4 + s] : 1u;
            if (cnt == 1u) {
                area_s = tt.area;
            } else {
                area_s = 0.0f;
                std::uint64_t const first = ref & k_qref_index_mask;
                for (std::uint32_t k = 0; k < cnt && first + k < p.primitive_count; ++k)
                    area_s += triangle_terms(p.triangles[first + k]).area;
            }
        } else {
            std::uint64_t const child = ref & k_qref_index_mask;
            area_s = child < p.node_count ? p.payload[child * p.payload_floats] : 0.0f;
        }
        if (area_s > 0.0f) {
            float const wgt = tt.area / area_s;
            dcx += wgt * hx;
            dcy += wgt * hy;
            dcz += wgt * hz;
            dA += (hx * dx + hy * dy + hz * dz) / area_s;
        }
        slot = p.parent_slot[node];
    }
    if (tt.area > 0.0f) {
        float const k = dA / tt.area;
        dnx += k * tt.nx;
        dny += k * tt.ny;
        dnz += k * tt.nz;
    }
    // n = (e1 x e2) / 2: dL/dv1 = (e2 x dn) / 2, dL/dv2 = (dn x e1) / 2, dL/dv0 = -(both)
    float const g1x = 0.5f * (tt.e2y * dnz - tt.e2z * dny);
    float const g1y = 0.5f * (tt.e2z * dnx - tt.e2x * dnz);
    float const g1z = 0.5f * (tt.e2x * dny - tt.e2y * dnx);
    float const g2x = 0.5f * (dny * tt.e1z - dnz * tt.e1y);
    float const g2y = 0.5f * (dnz * tt.e1x - dnx * tt.e1z);
    float const g2z = 0.5f * (dnx * tt.e1y - dny * tt.e1x);
    float const c3x = dcx / 3.0f, c3y = dcy / 3.0f, c3z = dcz / 3.0f;
    float const *ng = p.tri_grad + t * 9;
    float const v0x = -g1x - g2x + c3x + ng[0], v0y = -g1y - g2y + c3y + ng[1], v0z = -g1z - g2z + c3z + ng[2];
    float const v1x = g1x + c3x + ng[3], v1y = g1y + c3y + ng[4], v1z = g1z + c3z + ng[5];
    float const v2x = g2x + c3x + ng[6], v2y = g2y + c3y + ng[7], v2z = g2z + c3z + ng[8];
    std::uint32_t const prim = p.primitive_indices[t];
    if (prim >= p.g.triangle_count) {
        atomicOr(p.status, k_err_index);
        return;
    }
    std::uint32_t const i0 = p.g.tri_i0[prim], i1 = p.g.tri_i1[prim], i2 = p.g.tri_i2[prim];
    if (i0 >= p.g.vertex_count || i1 >= p.g.vertex_count || i2 >= p.g.vertex_count) {
        atomicOr(p.status, k_err_index);
        return;
    }
    atomicAdd(p.dvx + i0, v0x);
    atomicAdd(p.dvy + i0, v0y);
    atomicAdd(p.dvz + i0, v0z);
    atomicAdd(p.dvx + i1, v1x);
    atomicAdd(p.dvy + i1, v1y);
    atomicAdd(p.dvz + i1, v1z);
    atomicAdd(p.dvx + i2, v2x);
    atomicAdd(p.dvy + i2, v2y);
    atomicAdd(p.dvz + i2, v2z);
}

inline unsigned grid_for(std::uint64_t n, int block = 256) {
    return static_cast<unsigned>((n + block - 1) / block);
}

template <int Order>
int launch_traverse(adjoint_params const &p, int cap, int block, cudaStream_t s) {
    unsigned const grid = grid_for(p.n, block);
    if (cap <= 32)
        note_launch(), k_adjoint_traverse<Order, 32><<<grid, block, 0, s>>>(p);
    else
        note_launch(), k_adjoint_traverse<Order, 64><<<grid, block, 0, s>>>(p);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

} // namespace

int taylor_adjoint(adjoint_request const &r, cudaStream_t s) {
    bool const want_v = r.dvx != nullptr;
    std::uint64_t const nn = r.node_count, nt = r.primitive_count;
    int const sf = r.order == 0 ? slot_floats<0>::value : slot_floats<1>::value;
    if (want_v) {
        GWNB_CUDA_TRY(cudaMemsetAsync(r.dvx, 0, r.g.vertex_count * sizeof(float), s));
        GWNB_CUDA_TRY(cudaMemsetAsync(r.dvy, 0, r.g.vertex_count * sizeof(float), s));
        GWNB_CUDA_TRY(cudaMemsetAsync(r.dvz, 0, r.g.vertex_count * sizeof(float), s));
    }
    if (r.n == 0)
        return GWNB_OK;
    float *slot_grad = nullptr, *tri_grad = nullptr;
    std::uint32_t *order = nullptr, *tri_slot = nullptr;
    int rc = GWNB_OK;
    auto fail = [&](int code) {
        release(slot_grad, s);
        release(tri_grad, s);
        release(order, s);
        release(tri_slot, s);
        return code;
    };
    if (want_v) {
        if ((rc = alloc(&slot_grad, std::max<std::uint64_t>(nn * 4 * sf, 1), s)) != GWNB_OK)
            return fail(rc);
        if ((rc = alloc(&tri_grad, nt * 9, s)) != GWNB_OK)
            return fail(rc);
        if (cudaMemsetAsync(slot_grad, 0, std::max<std::uint64_t>(nn * 4 * sf, 1) * sizeof(float), s) != cudaSuccess ||
            cudaMemsetAsync(tri_grad, 0, nt * 9 * sizeof(float), s) != cudaSuccess)
            return fail(set_cuda_error(cudaGetLastError(), "adjoint scratch clear"));
    }
    if (r.sort_queries != 0 && r.n > 1 && r.root_bounds != nullptr) {
        if ((rc = alloc(&order, r.n, s)) != GWNB_OK)
            return fail(rc);
        if ((rc = query_order(r.root_bounds, r.qx, r.qy, r.qz, r.n, order, s, r.status)) != GWNB_OK)
            return fail(rc);
    }
    adjoint_params p{};
    p.qnodes = r.qnodes;
    p.qcounts = r.qcounts;
    p.tri48 = r.tri48;
    p.primitive_count = nt;
    p.node_count = nn;
    p.root_ref = r.root_ref;
    p.qx = r.qx;
    p.qy = r.qy;
    p.qz = r.qz;
    p.order = order;
    p.grad_out = r.grad_out;
    p.dqx = r.dqx;
    p.dqy = r.dqy;
    p.dqz = r.dqz;
    p.slot_grad = slot_grad;
    p.tri_grad = tri_grad;
    p.n = r.n;
    p.beta2 = r.accuracy_scale * r.accuracy_scale;
    p.status = r.status;
    int const block = query_launch_block(r.block);
    rc = r.order == 0 ? launch_traverse<0>(p, r.stack_capacity, block, s)
                      : launch_traverse<1>(p, r.stack_capacity, block, s);
    if (rc != GWNB_OK)
        return fail(rc);
    if (want_v) {
        if (nn > 0) {
            if ((rc = alloc(&tri_slot, nt, s)) != GWNB_OK)
                return fail(rc);
            if (cudaMemsetAsync(tri_slot, 0xff, nt * sizeof(std::uint32_t), s) != cudaSuccess)
                return fail(set_cuda_error(cudaGetLastError(), "adjoint leaf slots"));
            note_launch(), k_leaf_slots<<<grid_for(nn), 256, 0, s>>>(r.nodes, nn, nt, tri_slot);
        }
        adjoint_tri_params tp{};
        tp.qnodes = r.qnodes;
        tp.qcounts = r.qcounts;
        tp.triangles = r.triangles;
        tp.primitive_count = nt;
        tp.node_count = nn;
        tp.tri_slot = tri_slot;
        tp.parent_slot = r.parent_slot;
        tp.payload = r.payload;
        tp.payload_floats = r.payload_floats;
        tp.slot_grad = slot_grad;
        tp.tri_grad = tri_grad;
        tp.primitive_indices = r.primitive_indices;
        tp.g = r.g;
        tp.dvx = r.dvx;
        tp.dvy = r.dvy;
        tp.dvz = r.dvz;
        tp.status = r.status;
        if (r.order == 0)
            note_launch(), k_adjoint_triangles<0><<<grid_for(nt), 256, 0, s>>>(tp);
        else
            note_launch(), k_adjoint_triangles<1><<<grid_for(nt), 256, 0, s>>>(tp);
        cudaError_t const e = cudaGetLastError();
        if (e != cudaSuccess)
            return fail(set_cuda_error(e, "adjoint triangle pass"));
    }
    return fail(GWNB_OK);
}

} // namespace gwnb
