// Bottom-up refit of BVH4 bounds / triangle records and of Taylor moments.
//
// smallgwn recomputes parent links on every call, climbs with one thread per leaf edge into a
// pending array, commits in a third kernel and synchronizes (detail/gwn_bvh_refit_impl.cuh:23-334,
// detail/gwn_bvh_refit_moment_impl.cuh:17-279). Here parent links, expected arrival counts and
// the list of leaf-bearing nodes are derived once per BVH and cached; each refit is one kernel in
// which one thread per leaf-bearing node refreshes its triangles, and the last arrival at a node
// (children in slot order) finishes it and climbs. The last arriver also zeroes the node's counter,
// so repeated refits need no memset and can be captured in a CUDA graph.
//
// Moment arithmetic restates smallgwn's (detail/gwn_bvh_refit_common.cuh):
//   per-triangle raw moments :123-387 (area, area*centroid, N = 1/2 e1 x e2, N (x) centroid, and
//   for order 2 the sorted-vertex split integrals of the SideFX HDK UT_SolidAngle);
//   accumulation :67-111 (first valid child, then the others in slot order);
//   recentring and coefficient packing :514-608; far-field radius :113-121.
#include "gwnb_internal.cuh"

#include <new>
#include <vector>

namespace gwnb {
namespace {

constexpr int k_block = 128;

// ---- aux preparation ---------------------------------------------------------------------------

// summary, when non-null, is a build's device-side collapse summary (the build has not read it back
// yet and launches over its node capacity): its node count bounds the nodes, and a collapse that
// has not reached the bottom of the tree yet (pending) leaves nothing to derive.
__global__ void __launch_bounds__(256)
    k_prepare_aux(node4 const *__restrict__ nodes, std::uint64_t node_count,
                  std::uint64_t primitive_count, std::uint32_t *__restrict__ parent_slot,
                  std::uint32_t *__restrict__ expected, std::uint32_t *__restrict__ leaf_nodes,
                  std::uint32_t *leaf_node_counter, unsigned int *status, collapse_summary const *summary) {
    if (summary != nullptr) {
        if (summary->pending != 0u)
            return;
        if (summary->node_count < node_count)
            node_count = summary->node_count;
    }
    std::uint64_t const n = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= node_count)
        return;
    std::uint32_t k_int = 0;
    bool has_leaf = false;
    bool any = false;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        std::uint64_t const r = nodes[n].c[s].reference;
        if (!ref_valid(r))
            continue;
        any = true;
        if (ref_internal(r)) {
            std::uint64_t const c = ref_offset(r);
            if (c >= node_count || c == 0) {
                atomicOr(status, k_err_topology);
                continue;
            }
            parent_slot[c] = static_cast<std::uint32_t>((n << 2) | static_cast<std::uint64_t>(s));
            ++k_int;
        } else {
            std::uint64_t const b = ref_offset(r);
            std::uint64_t const cnt = ref_count(r);
            if (b > primitive_count || cnt > primitive_count - b)
                atomicOr(status, k_err_topology);
            has_leaf = true;
        }
    }
    if (!any)
        atomicOr(status, k_err_topology);
    expected[n] = k_int + (has_leaf ? 1u : 0u);
    if (has_leaf)
        leaf_nodes[atomicAdd(leaf_node_counter, 1u)] = static_cast<std::uint32_t>(n);
}

// ---- bounds refit ------------------------------------------------------------------------------

struct tri_payload {
    triangle t;
    aabb b;
    bool valid;
};

__device__ inline tri_payload make_triangle(gwnb_geometry_f32 const &g, std::uint32_t prim) {
    tri_payload r{};
    r.valid = false;
    if (prim >= g.triangle_count)
        return r;
    std::uint32_t const a = g.tri_i0[prim], b = g.tri_i1[prim], c = g.tri_i2[prim];
    std::uint64_t const nv = g.vertex_count;
    if (a >= nv || b >= nv || c >= nv)
        return r;
    float const v0x = g.vertex_x[a], v0y = g.vertex_y[a], v0z = g.vertex_z[a];
    float const v1x = g.vertex_x[b], v1y = g.vertex_y[b], v1z = g.vertex_z[b];
    float const v2x = g.vertex_x[c], v2y = g.vertex_y[c], v2z = g.vertex_z[c];
    r.t = triangle{v0x, v0y, v0z, __fsub_rn(v1x, v0x), __fsub_rn(v1y, v0y), __fsub_rn(v1z, v0z),
                   __fsub_rn(v2x, v0x), __fsub_rn(v2y, v0y), __fsub_rn(v2z, v0z)};
    r.b = aabb{rmin(v0x, rmin(v1x, v2x)), rmin(v0y, rmin(v1y, v2y)), rmin(v0z, rmin(v1z, v2z)),
               rmax(v0x, rmax(v1x, v2x)), rmax(v0y, rmax(v1y, v2y)), rmax(v0z, rmax(v1z, v2z))};
    r.valid = true;
    return r;
}

__device__ inline void store_tri(triangle *tris, triangle48 *tri48, std::uint64_t i, triangle const &t) {
    tris[i] = t;
    if (tri48 != nullptr)
        tri48[i] = make_triangle48(t.v0_x, t.v0_y, t.v0_z, t.e1_x, t.e1_y, t.e1_z, t.e2_x, t.e2_y, t.e2_z);
}

__device__ inline aabb load_bounds_cg(node4 const *nodes, std::uint64_t n, int s) {
    float const *p = reinterpret_cast<float const *>(&nodes[n].c[s].bounds);
    return aabb{__ldcg(p), __ldcg(p + 1), __ldcg(p + 2), __ldcg(p + 3), __ldcg(p + 4), __ldcg(p + 5)};
}

struct refit_params {
    gwnb_geometry_f32 g;
    node4 *nodes;
    std::uint64_t node_count;
    std::uint32_t const *primitive_indices;
    triangle *triangles;
    triangle48 *tri48;
    std::uint64_t primitive_count;
    std::uint32_t const *parent_slot;
    std::uint32_t const *expected;
    std::uint32_t *arrivals;
    std::uint32_t const *leaf_nodes;
    std::uint64_t leaf_node_count;
    aabb *root_bounds;
    unsigned int *status;
};

// One work item of the bounds refit: leaf-bearing node t of the BVH refreshes its triangles, then
// climbs while it is the last arrival.
__device__ __forceinline__ void refit_bounds_item(refit_params const &p, std::uint64_t t) {
    std::uint32_t cur = p.leaf_nodes[t];
    // Refresh the leaf children of this node.
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        std::uint64_t const r = p.nodes[cur].c[s].reference;
        if (!ref_leaf(r))
            continue;
        std::uint64_t const first = ref_offset(r);
        std::uint32_t const cnt = ref_count(r);
        aabb u{0, 0, 0, 0, 0, 0};
        bool init = false;
        for (std::uint32_t k = 0; k < cnt; ++k) {
            std::uint64_t const si = first + k;
            if (si >= p.primitive_count) {
                atomicOr(p.status, k_err_topology);
                break;
            }
            tri_payload const tp = make_triangle(p.g, p.primitive_indices[si]);
            if (!tp.valid) {
                atomicOr(p.status, k_err_index);
                continue;
            }
            store_tri(p.triangles, p.tri48, si, tp.t);
            u = init ? aabb_union(u, tp.b) : tp.b;
            init = true;
        }
        p.nodes[cur].c[s].bounds = u;
    }
    // Climb: the last arrival at a node unions its children and continues to the parent.
    std::uint64_t guard = 0;
    for (;;) {
        fence_acq_rel_gpu();
        std::uint32_t const arrived = atomicAdd(&p.arrivals[cur], 1u) + 1u;
        std::uint32_t const expect = p.expected[cur];
        if (arrived < expect)
            return;
        if (arrived > expect) {
            atomicOr(p.status, k_err_topology);
            return;
        }
        p.arrivals[cur] = 0u;
        fence_acq_rel_gpu();
        aabb u{0, 0, 0, 0, 0, 0};
        bool init = false;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            std::uint64_t const r = __ldcg(reinterpret_cast<unsigned long long const *>(&p.nodes[cur].c[s].reference));
            if (!ref_valid(r))
                continue;
            aabb const b = load_bounds_cg(p.nodes, cur, s);
            u = init ? aabb_union(u, b) : b;
            init = true;
        }
        std::uint32_t const ps = p.parent_slot[cur];
        if (ps == k_invalid_u32) {
            *p.root_bounds = u;
            return;
        }
        std::uint32_t const parent = ps >> 2;
        if (parent >= p.node_count || ++guard > p.node_count) {
            atomicOr(p.status, k_err_topology);
            return;
        }
        p.nodes[parent].c[ps & 3u].bounds = u;
        cur = parent;
    }
}

__global__ void __launch_bounds__(k_block) k_refit_bounds(refit_params p) {
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < p.leaf_node_count)
        refit_bounds_item(p, t);
}

// The whole refit of a BVH whose root is a leaf (one work item).
__device__ __forceinline__ void refit_leaf_root_item(refit_params const &p, std::uint64_t first, std::uint32_t cnt) {
    aabb u{0, 0, 0, 0, 0, 0};
    bool init = false;
    for (std::uint32_t k = 0; k < cnt; ++k) {
        std::uint64_t const si = first + k;
        if (si >= p.primitive_count) {
            atomicOr(p.status, k_err_topology);
            break;
        }
        tri_payload const tp = make_triangle(p.g, p.primitive_indices[si]);
        if (!tp.valid) {
            atomicOr(p.status, k_err_index);
            continue;
        }
        store_tri(p.triangles, p.tri48, si, tp.t);
        u = init ? aabb_union(u, tp.b) : tp.b;
        init = true;
    }
    *p.root_bounds = u;
}

__global__ void k_refit_leaf_root(refit_params p, std::uint64_t first, std::uint32_t cnt) {
    refit_leaf_root_item(p, first, cnt);
}

// ---- moments -----------------------------------------------------------------------------------

template <int Order> struct payload;
template <> struct payload<0> {
    float area, apx, apy, apz, nx, ny, nz;
};
template <> struct payload<1> : payload<0> {
    float nxx, nxy, nxz, nyx, nyy, nyz, nzx, nzy, nzz; // n_i * centroid_j
};
template <> struct payload<2> : payload<1> {
    float r[3][6]; // raw second moments per normal component i over jk in {xx,yy,zz,xy,yz,zx}
};

template <int Order> __device__ inline void accumulate(payload<Order> &d, payload<Order> const &s) {
    d.area += s.area;
    d.apx += s.apx;
    d.apy += s.apy;
    d.apz += s.apz;
    d.nx += s.nx;
    d.ny += s.ny;
    d.nz += s.nz;
    if constexpr (Order >= 1) {
        d.nxx += s.nxx;
        d.nxy += s.nxy;
        d.nxz += s.nxz;
        d.nyx += s.nyx;
        d.nyy += s.nyy;
        d.nyz += s.nyz;
        d.nzx += s.nzx;
        d.nzy += s.nzy;
        d.nzz += s.nzz;
    }
    if constexpr (Order >= 2) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 6; ++j)
                d.r[i][j] += s.r[i][j];
    }
}

// Area-weighted integrals of (p - P)_i (p - P)_j over a triangle, by splitting it at the middle
// vertex along axis i (SideFX HDK UT_SolidAngle). v = vertices sorted along axis i; writes the
// ii integral and optionally the ij / ik cross integrals.
__device__ inline void split_integrals(float const (&vs)[3][3], int va, int vb, int vc, int i,
                                       float const (&P)[3], float *out_ii, float *out_ij,
                                       float *out_ik) {
    int const j = (i == 2) ? 0 : i + 1;
    int const k = (j == 2) ? 0 : j + 1;
    float const oab_i = vs[vb][i] - vs[va][i];
    float const oab_j = vs[vb][j] - vs[va][j];
    float const oab_k = vs[vb][k] - vs[va][k];
    float const oac_i = vs[vc][i] - vs[va][i];
    float const oac_j = vs[vc][j] - vs[va][j];
    float const oac_k = vs[vc][k] - vs[va][k];
    float const ocb_i = vs[vb][i] - vs[vc][i];
    float const ocb_j = vs[vb][j] - vs[vc][j];
    float const ocb_k = vs[vb][k] - vs[vc][k];
    float const t = (oac_i > 0.0f) ? (oab_i / oac_i) : 0.0f;
    float const jd = t * oac_j - oab_j;
    float const kd = t * oac_k - oab_k;
    float const ca0 = jd * oab_k - kd * oab_j;
    float const ca1 = kd * oab_i;
    float const ca2 = jd * oab_i;
    float const cc0 = jd * ocb_k - kd * ocb_j;
    float const cc1 = kd * ocb_i;
    float const cc2 = jd * ocb_i;
    float const sa = sqrtf(rmax(ca0 * ca0 + ca1 * ca1 + ca2 * ca2, 0.0f));
    float const sc = sqrtf(rmax(cc0 * cc0 + cc1 * cc1 + cc2 * cc2, 0.0f));
    float const pai = vs[va][i] - P[i];
    float const pci = vs[vc][i] - P[i];
    *out_ii = sa * (0.5f * pai * pai + (2.0f / 3.0f) * pai * oab_i + 0.25f * oab_i * oab_i) +
              sc * (0.5f * pci * pci + (2.0f / 3.0f) * pci * ocb_i + 0.25f * ocb_i * ocb_i);
    auto cross = [&](int jk, float diff, float *out) {
        if (out == nullptr)
            return;
        float const mid = vs[vb][jk] + 0.5f * diff;
        float const amid = mid - vs[va][jk];
        float const cmid = mid - vs[vc][jk];
        float const paj = vs[va][jk] - P[jk];
        float const pcj = vs[vc][jk] - P[jk];
        *out = sa * (0.5f * pai * paj + (1.0f / 3.0f) * pai * amid + (1.0f / 3.0f) * paj * oab_i +
                     0.25f * oab_i * amid) +
               sc * (0.5f * pci * pcj + (1.0f / 3.0f) * pci * cmid + (1.0f / 3.0f) * pcj * ocb_i +
                     0.25f * ocb_i * cmid);
    };
    cross(j, jd, out_ij);
    cross(k, kd, out_ik);
}

template <int Order> __device__ inline payload<Order> triangle_moment(triangle const &t) {
    payload<Order> m{};
    float const ax = t.v0_x, ay = t.v0_y, az = t.v0_z;
    float const bx = ax + t.e1_x, by = ay + t.e1_y, bz = az + t.e1_z;
    float const cx = ax + t.e2_x, cy = ay + t.e2_y, cz = az + t.e2_z;
    float const px = (ax + bx + cx) / 3.0f;
    float const py = (ay + by + cy) / 3.0f;
    float const pz = (az + bz + cz) / 3.0f;
    float const abx = bx - ax, aby = by - ay, abz = bz - az;
    float const acx = cx - ax, acy = cy - ay, acz = cz - az;
    float const nx = 0.5f * (aby * acz - abz * acy);
    float const ny = 0.5f * (abz * acx - abx * acz);
    float const nz = 0.5f * (abx * acy - aby * acx);
    float const area = sqrtf(rmax(nx * nx + ny * ny + nz * nz, 0.0f));
    m.area = area;
    m.apx = px * area;
    m.apy = py * area;
    m.apz = pz * area;
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    if constexpr (Order >= 1) {
        m.nxx = nx * px;
        m.nxy = nx * py;
        m.nxz = nx * pz;
        m.nyx = ny * px;
        m.nyy = ny * py;
        m.nyz = ny * pz;
        m.nzx = nz * px;
        m.nzy = nz * py;
        m.nzz = nz * pz;
    }
    if constexpr (Order >= 2) {
        if (area == 0.0f)
            return m; // zero-area triangles contribute no second moments
        float const inv_area = 1.0f / area;
        float const nh[3] = {nx * inv_area, ny * inv_area, nz * inv_area};
        float const vs[3][3] = {{ax, ay, az}, {bx, by, bz}, {cx, cy, cz}};
        float const P[3] = {px, py, pz};
        int ord[3][3];
        float span[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int o0 = 0, o1 = 1, o2 = 2, tmp;
            if (vs[0][a] > vs[1][a]) {
                tmp = o0; o0 = o1; o1 = tmp;
            }
            if (vs[o0][a] > vs[2][a]) {
                tmp = o0; o0 = o2; o2 = tmp;
            }
            if (vs[o1][a] > vs[o2][a]) {
                tmp = o1; o1 = o2; o2 = tmp;
            }
            ord[a][0] = o0;
            ord[a][1] = o1;
            ord[a][2] = o2;
            span[a] = vs[o2][a] - vs[o0][a];
        }
        float ixx = 0, iyy = 0, izz = 0, ixy = 0, iyz = 0, izx = 0;
        float const dx = span[0], dy = span[1], dz = span[2];
        if (dx > 0.0f)
            split_integrals(vs, ord[0][0], ord[0][1], ord[0][2], 0, P, &ixx,
                            (dx >= dy && dy > 0.0f) ? &ixy : nullptr,
                            (dx >= dz && dz > 0.0f) ? &izx : nullptr);
        if (dy > 0.0f)
            split_integrals(vs, ord[1][0], ord[1][1], ord[1][2], 1, P, &iyy,
                            (dy >= dz && dz > 0.0f) ? &iyz : nullptr,
                            (dx < dy && dx > 0.0f) ? &ixy : nullptr);
        if (dz > 0.0f)
            split_integrals(vs, ord[2][0], ord[2][1], ord[2][2], 2, P, &izz,
                            (dx < dz && dx > 0.0f) ? &izx : nullptr,
                            (dy < dz && dy > 0.0f) ? &iyz : nullptr);
        float const ig[6] = {ixx, iyy, izz, ixy, iyz, izx};
        float const N[3] = {nx, ny, nz};
        float const pp[6] = {px * px, py * py, pz * pz, px * py, py * pz, pz * px};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 6; ++j)
                m.r[i][j] = nh[i] * ig[j] + N[i] * pp[j];
    }
    return m;
}

// Coefficients of one child slot: smallgwn's field order per moment node.
template <int Order> struct coeffs {
    float f[Order == 0 ? 7 : (Order == 1 ? 13 : 23)];
};

template <int Order>
__device__ inline coeffs<Order> finalize_slot(aabb const &b, payload<Order> const &m) {
    coeffs<Order> c{};
    float ax, ay, az;
    if (m.area > 0.0f) {
        ax = m.apx / m.area;
        ay = m.apy / m.area;
        az = m.apz / m.area;
    } else {
        ax = (b.min_x + b.max_x) * 0.5f;
        ay = (b.min_y + b.max_y) * 0.5f;
        az = (b.min_z + b.max_z) * 0.5f;
    }
    float const dx = rmax(ax - b.min_x, b.max_x - ax);
    float const dy = rmax(ay - b.min_y, b.max_y - ay);
    float const dz = rmax(az - b.min_z, b.max_z - az);
    c.f[0] = dx * dx + dy * dy + dz * dz;
    c.f[1] = ax;
    c.f[2] = ay;
    c.f[3] = az;
    c.f[4] = m.nx;
    c.f[5] = m.ny;
    c.f[6] = m.nz;
    if constexpr (Order >= 1) {
        float const xx = m.nxx - ax * m.nx;
        float const yy = m.nyy - ay * m.ny;
        float const zz = m.nzz - az * m.nz;
        float const xy = m.nxy - ay * m.nx;
        float const yx = m.nyx - ax * m.ny;
        float const yz = m.nyz - az * m.ny;
        float const zy = m.nzy - ay * m.nz;
        float const zx = m.nzx - ax * m.nz;
        float const xz = m.nxz - az * m.nx;
        c.f[7] = xx;
        c.f[8] = yy;
        c.f[9] = zz;
        c.f[10] = xy + yx;
        c.f[11] = yz + zy;
        c.f[12] = zx + xz;
    }
    if constexpr (Order >= 2) {
        float const P[3] = {ax, ay, az};
        float const N[3] = {m.nx, m.ny, m.nz};
        // first moments F_i_j = n_i * centroid_j summed
        float const F[3][3] = {{m.nxx, m.nxy, m.nxz}, {m.nyx, m.nyy, m.nyz}, {m.nzx, m.nzy, m.nzz}};
        // centred_i_jk = raw_i_jk - P_j F_i_k - P_k F_i_j + P_j P_k N_i ; jk in {xx,yy,zz,xy,yz,zx}
        float cen[3][6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            cen[i][0] = m.r[i][0] - 2.0f * P[0] * F[i][0] + P[0] * P[0] * N[i];
            cen[i][1] = m.r[i][1] - 2.0f * P[1] * F[i][1] + P[1] * P[1] * N[i];
            cen[i][2] = m.r[i][2] - 2.0f * P[2] * F[i][2] + P[2] * P[2] * N[i];
            cen[i][3] = m.r[i][3] - P[0] * F[i][1] - P[1] * F[i][0] + P[0] * P[1] * N[i];
            cen[i][4] = m.r[i][4] - P[1] * F[i][2] - P[2] * F[i][1] + P[1] * P[2] * N[i];
            cen[i][5] = m.r[i][5] - P[2] * F[i][0] - P[0] * F[i][2] + P[2] * P[0] * N[i];
        }
        c.f[13] = cen[0][0];                                   // Nxxx
        c.f[14] = cen[1][1];                                   // Nyyy
        c.f[15] = cen[2][2];                                   // Nzzz
        c.f[16] = 2.0f * (cen[0][4] + cen[1][5] + cen[2][3]);  // sum of Nxyz permutations
        c.f[17] = 2.0f * cen[0][3] + cen[1][0];                // 2Nxxy + Nyxx
        c.f[18] = 2.0f * cen[0][5] + cen[2][0];                // 2Nxxz + Nzxx
        c.f[19] = 2.0f * cen[1][4] + cen[2][1];                // 2Nyyz + Nzyy
        c.f[20] = 2.0f * cen[1][3] + cen[0][1];                // 2Nyyx + Nxyy
        c.f[21] = 2.0f * cen[2][5] + cen[0][2];                // 2Nzzx + Nxzz
        c.f[22] = 2.0f * cen[2][4] + cen[1][2];                // 2Nzzy + Nyzz
    }
    return c;
}

// Sidecar coefficients of the far-field terms, folded for the traversal (the reference layout keeps
// smallgwn's fields). With n = r / |r| a unit vector, smallgwn's order-1 term (T - 3S) / |r|^3
// (T = tr M, S = n^T M n) is the single quadratic form n^T M' n, M' = T I - 3 M; its order-2 term
// (1.5 n.V - 7.5 C(n,n,n)) / |r|^4 (V_x = 3 N_xxx + A_yx + A_zx and cyclically) becomes, since
// n.V = (n.V)(n.n), the single cubic form K(n,n,n). Written: order 1 the 6 coefficients of M' over
// xx yy zz xy yz zx; order 2 the 10 of K over xxx yyy zzz xxy xxz yyx yyz zzx zzy xyz.
template <int Order>
__device__ inline void fold_far_field_coefficients(coeffs<Order> const &c, float *out) {
    float const T = c.f[7] + c.f[8] + c.f[9];
    out[0] = T - 3.0f * c.f[7];
    out[1] = T - 3.0f * c.f[8];
    out[2] = T - 3.0f * c.f[9];
    out[3] = -3.0f * c.f[10];
    out[4] = -3.0f * c.f[11];
    out[5] = -3.0f * c.f[12];
    if constexpr (Order >= 2) {
        float const xxx = c.f[13], yyy = c.f[14], zzz = c.f[15], spn = c.f[16];
        float const Axy = c.f[17], Axz = c.f[18], Ayz = c.f[19], Ayx = c.f[20], Azx = c.f[21], Azy = c.f[22];
        float const vx = 1.5f * (3.0f * xxx + Ayx + Azx);
        float const vy = 1.5f * (3.0f * yyy + Azy + Axy);
        float const vz = 1.5f * (3.0f * zzz + Axz + Ayz);
        out[6] = vx - 7.5f * xxx;
        out[7] = vy - 7.5f * yyy;
        out[8] = vz - 7.5f * zzz;
        out[9] = vy - 7.5f * Axy;
        out[10] = vz - 7.5f * Axz;
        out[11] = vx - 7.5f * Ayx;
        out[12] = vz - 7.5f * Ayz;
        out[13] = vx - 7.5f * Azx;
        out[14] = vy - 7.5f * Azy;
        out[15] = -7.5f * spn;
    }
}

struct moment_params {
    node4 const *nodes;
    std::uint64_t node_count;
    triangle const *triangles;
    std::uint64_t primitive_count;
    std::uint32_t const *parent_slot;
    std::uint32_t const *expected;
    std::uint32_t *arrivals;
    std::uint32_t const *leaf_nodes;
    std::uint64_t leaf_node_count;
    float *ref_nodes;      // smallgwn field-SoA moment nodes
    float4 *qnodes;        // query sidecar
    std::uint32_t *qcounts;
    void *pending;         // per-node payload
    unsigned int *status;
};

template <int Order> __device__ inline void store_payload_cg(payload<Order> *dst, payload<Order> const &v) {
    float const *s = reinterpret_cast<float const *>(&v);
    float *d = reinterpret_cast<float *>(dst);
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(payload<Order>) / 4); ++k)
        __stcg(d + k, s[k]);
}
template <int Order> __device__ inline payload<Order> load_payload_cg(payload<Order> const *src) {
    payload<Order> v;
    float const *s = reinterpret_cast<float const *>(src);
    float *d = reinterpret_cast<float *>(&v);
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(payload<Order>) / 4); ++k)
        d[k] = __ldcg(s + k);
    return v;
}

template <int Order>
__device__ inline void finish_node(moment_params const &p, std::uint32_t n) {
    constexpr int F = Order == 0 ? 7 : (Order == 1 ? 13 : 23);
    constexpr int Q = qnode_traits<Order>::k_f4_per_child;
    payload<Order> *pend = static_cast<payload<Order> *>(p.pending);
    payload<Order> total{};
    bool init = false;
    float *ref = p.ref_nodes + static_cast<std::uint64_t>(n) * F * 4;
    float4 *qn = p.qnodes + static_cast<std::uint64_t>(n) * 4 * Q;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        node4 const &nd = p.nodes[n];
        std::uint64_t const r = nd.c[s].reference;
        float q[Q * 4];
#pragma unroll
        for (int k = 0; k < Q * 4; ++k)
            q[k] = 0.0f;
        if (!ref_valid(r)) {
#pragma unroll
            for (int f = 0; f < F; ++f)
                ref[f * 4 + s] = 0.0f;
            q[3] = -1.0f;
            q[7] = __uint_as_float(k_invalid_u32);
            p.qcounts[n * 4 + s] = 0u;
        } else {
            payload<Order> m{};
            std::uint32_t qref = 0;
            if (ref_internal(r)) {
                std::uint64_t const c = ref_offset(r);
                if (c < p.node_count)
                    m = load_payload_cg(pend + c);
                else
                    atomicOr(p.status, k_err_topology);
                qref = static_cast<std::uint32_t>(c) & k_qref_index_mask;
                p.qcounts[n * 4 + s] = 0u;
            } else {
                std::uint64_t const first = ref_offset(r);
                std::uint32_t const cnt = ref_count(r);
                for (std::uint32_t k = 0; k < cnt; ++k) {
                    std::uint64_t const si = first + k;
                    if (si >= p.primitive_count) {
                        atomicOr(p.status, k_err_topology);
                        break;
                    }
                    payload<Order> const tm = triangle_moment<Order>(p.triangles[si]);
                    if (k == 0)
                        m = tm;
                    else
                        accumulate(m, tm);
                }
                qref = k_qref_leaf | (static_cast<std::uint32_t>(first) & k_qref_index_mask) |
                       (cnt > 1 ? k_qref_multi : 0u);
                p.qcounts[n * 4 + s] = cnt;
            }
            aabb const b = load_bounds_cg(p.nodes, n, s);
            coeffs<Order> const c = finalize_slot<Order>(b, m);
#pragma unroll
            for (int f = 0; f < F; ++f)
                ref[f * 4 + s] = c.f[f];
            // sidecar: a = (P, r2), b = (N, ref), then coefficients 7.. in order
            q[0] = c.f[1];
            q[1] = c.f[2];
            q[2] = c.f[3];
            q[3] = c.f[0];
            q[4] = c.f[4];
            q[5] = c.f[5];
            q[6] = c.f[6];
            q[7] = __uint_as_float(qref);
            if constexpr (Order >= 1)
                fold_far_field_coefficients<Order>(c, q + 8);
            if (init)
                accumulate(total, m);
            else
                total = m;
            init = true;
        }
#pragma unroll
        for (int k = 0; k < Q; ++k)
            qn[s * Q + k] = make_float4(q[4 * k], q[4 * k + 1], q[4 * k + 2], q[4 * k + 3]);
    }
    store_payload_cg(pend + n, total);
}

// One work item of the moment refit: from leaf-bearing node t, finish every node this thread is
// the last arrival at, climbing to the root.
template <int Order> __device__ __forceinline__ void refit_moments_item(moment_params const &p, std::uint64_t t) {
    std::uint32_t cur = p.leaf_nodes[t];
    std::uint64_t guard = 0;
    for (;;) {
        fence_acq_rel_gpu();
        std::uint32_t const arrived = atomicAdd(&p.arrivals[cur], 1u) + 1u;
        std::uint32_t const expect = p.expected[cur];
        if (arrived < expect)
            return;
        if (arrived > expect) {
            atomicOr(p.status, k_err_topology);
            return;
        }
        p.arrivals[cur] = 0u;
        fence_acq_rel_gpu();
        finish_node<Order>(p, cur);
        std::uint32_t const ps = p.parent_slot[cur];
        if (ps == k_invalid_u32)
            return;
        std::uint32_t const parent = ps >> 2;
        if (parent >= p.node_count || ++guard > p.node_count) {
            atomicOr(p.status, k_err_topology);
            return;
        }
        cur = parent;
    }
}

template <int Order> __global__ void __launch_bounds__(k_block) k_refit_moments(moment_params p) {
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < p.leaf_node_count)
        refit_moments_item<Order>(p, t);
}

// ---- batched refit (many BVHs, one launch) -------------------------------------------------------
//
// Mesh m owns work items [begin[m], begin[m + 1]) of a global index space: its leaf-bearing nodes,
// or a single item when its root is a leaf. A persistent grid strides over the items; each finds its
// mesh by binary search over `begin` (mesh_count + 1 ascending offsets) and runs the single-BVH item.
// The climbs never wait on one another (the last arrival continues), so any grid size is safe.

__device__ __forceinline__ std::uint32_t find_mesh(std::uint64_t const *begin, std::uint32_t mesh_count,
                                                   std::uint64_t item) {
    std::uint32_t lo = 0, hi = mesh_count; // begin[lo] <= item < begin[hi]
    while (hi - lo > 1) {
        std::uint32_t const mid = (lo + hi) >> 1;
        if (__ldg(begin + mid) <= item)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

struct batch_bounds_mesh {
    refit_params p;
    std::uint64_t leaf_root_first; // root is a leaf: its triangle range (leaf_root_count > 0)
    std::uint32_t leaf_root_count;
};

constexpr int k_batch_block_max = 256; // batched refit launches take 32..256 threads per block

__global__ void __launch_bounds__(k_batch_block_max)
    k_batch_refit_bounds(batch_bounds_mesh const *__restrict__ meshes, std::uint64_t const *__restrict__ begin,
                         std::uint32_t mesh_count) {
    std::uint64_t const total = begin[mesh_count];
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        std::uint32_t const m = find_mesh(begin, mesh_count, i);
        batch_bounds_mesh const &d = meshes[m];
        if (d.leaf_root_count > 0)
            refit_leaf_root_item(d.p, d.leaf_root_first, d.leaf_root_count);
        else
            refit_bounds_item(d.p, i - begin[m]);
    }
}

template <int Order>
__global__ void __launch_bounds__(k_batch_block_max)
    k_batch_refit_moments(moment_params const *__restrict__ meshes, std::uint64_t const *__restrict__ begin,
                          std::uint32_t mesh_count) {
    std::uint64_t const total = begin[mesh_count];
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        std::uint32_t const m = find_mesh(begin, mesh_count, i);
        refit_moments_item<Order>(meshes[m], i - begin[m]);
    }
}

inline unsigned grid_for(std::uint64_t n, int block = k_block) {
    return static_cast<unsigned>((n + block - 1) / block);
}

} // namespace

// ---- host ---------------------------------------------------------------------------------------

int create_bvh_aux(gwnb_bvh4_f32 *bvh, cudaStream_t s) {
    if (bvh->aux != nullptr)
        return GWNB_OK;
    auto *a = new (std::nothrow) bvh_aux_impl{};
    if (a == nullptr)
        return set_error(GWNB_INTERNAL_ERROR, "out of host memory");
    a->stream = s;
    bvh->aux = reinterpret_cast<gwnb_bvh_aux *>(a);
    GWNB_TRY(alloc(&a->status, 1, s));
    GWNB_TRY(alloc(&a->root_bounds, 1, s));
    GWNB_TRY(alloc(&a->fp64_count, 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(a->status, 0, sizeof(unsigned int), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(a->fp64_count, 0, sizeof(unsigned long long), s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(a->root_bounds, &bvh->root.bounds, sizeof(aabb), cudaMemcpyHostToDevice, s));
    return GWNB_OK;
}

int ensure_bvh_aux(gwnb_bvh4_f32 *bvh, cudaStream_t s) {
    GWNB_TRY(create_bvh_aux(bvh, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    bool const fresh = a->derived && a->nodes_ptr == bvh->nodes && a->triangles_ptr == bvh->triangles &&
                       a->node_count == bvh->node_count && a->primitive_count == bvh->primitive_count &&
                       a->revision == bvh->revision;
    if (fresh)
        return GWNB_OK;
    release(a->parent_slot, s);
    release(a->expected, s);
    release(a->arrivals, s);
    release(a->leaf_nodes, s);
    release(a->tri48, s);
    a->leaf_node_count = 0;
    std::uint64_t const nn = bvh->node_count;
    GWNB_TRY(alloc(&a->tri48, bvh->primitive_count, s));
    if (nn > 0) {
        GWNB_TRY(alloc(&a->parent_slot, nn, s));
        GWNB_TRY(alloc(&a->expected, nn, s));
        GWNB_TRY(alloc(&a->arrivals, 2 * nn, s));
        GWNB_TRY(alloc(&a->leaf_nodes, nn + 1, s));
        GWNB_CUDA_TRY(cudaMemsetAsync(a->parent_slot, 0xff, nn * sizeof(std::uint32_t), s));
        GWNB_CUDA_TRY(cudaMemsetAsync(a->arrivals, 0, 2 * nn * sizeof(std::uint32_t), s));
        GWNB_CUDA_TRY(cudaMemsetAsync(a->leaf_nodes + nn, 0, sizeof(std::uint32_t), s));
        note_launch(), k_prepare_aux<<<grid_for(nn, 256), 256, 0, s>>>(
            reinterpret_cast<node4 const *>(bvh->nodes), nn, bvh->primitive_count, a->parent_slot,
            a->expected, a->leaf_nodes, a->leaf_nodes + nn, a->status, nullptr);
        GWNB_CUDA_TRY(cudaGetLastError());
        std::uint32_t count = 0;
        GWNB_CUDA_TRY(cudaMemcpyAsync(&count, a->leaf_nodes + nn, sizeof(count), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
        a->leaf_node_count = count;
    }
    GWNB_TRY(write_tri48(bvh, s));
    a->nodes_ptr = bvh->nodes;
    a->triangles_ptr = bvh->triangles;
    a->derived = true;
    a->node_count = nn;
    a->primitive_count = bvh->primitive_count;
    a->revision = bvh->revision;
    return GWNB_OK;
}

int prepare_bvh_aux_async(gwnb_bvh4_f32 *bvh, std::uint64_t cap, collapse_summary const *summary,
                          std::uint32_t *leaf_node_count, cudaStream_t s) {
    GWNB_TRY(create_bvh_aux(bvh, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    release(a->parent_slot, s);
    release(a->expected, s);
    release(a->arrivals, s);
    release(a->leaf_nodes, s);
    release(a->tri48, s);
    a->leaf_node_count = 0;
    a->derived = false;
    GWNB_TRY(alloc(&a->tri48, std::max<std::uint64_t>(bvh->primitive_count, 1), s));
    if (cap == 0)
        return GWNB_OK;
    GWNB_TRY(alloc(&a->parent_slot, cap, s));
    GWNB_TRY(alloc(&a->expected, cap, s));
    GWNB_TRY(alloc(&a->arrivals, 2 * cap, s));
    GWNB_TRY(alloc(&a->leaf_nodes, cap + 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(a->parent_slot, 0xff, cap * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(a->arrivals, 0, 2 * cap * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(a->leaf_nodes + cap, 0, sizeof(std::uint32_t), s));
    note_launch(), k_prepare_aux<<<grid_for(cap, 256), 256, 0, s>>>(
        reinterpret_cast<node4 const *>(bvh->nodes), cap, bvh->primitive_count, a->parent_slot, a->expected,
        a->leaf_nodes, a->leaf_nodes + cap, a->status, summary);
    GWNB_CUDA_TRY(cudaGetLastError());
    GWNB_CUDA_TRY(cudaMemcpyAsync(leaf_node_count, a->leaf_nodes + cap, sizeof(std::uint32_t), cudaMemcpyDeviceToDevice,
                                  s));
    return GWNB_OK;
}

namespace {
__global__ void k_tri48(triangle const *__restrict__ tris, triangle48 *__restrict__ out, std::uint64_t n) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        store_tri(const_cast<triangle *>(tris), out, i, tris[i]);
}
} // namespace

int write_tri48(gwnb_bvh4_f32 const *bvh, cudaStream_t s) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    if (bvh->primitive_count == 0)
        return GWNB_OK;
    note_launch(), k_tri48<<<grid_for(bvh->primitive_count, 256), 256, 0, s>>>(
        reinterpret_cast<triangle const *>(bvh->triangles), a->tri48, bvh->primitive_count);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

namespace {
refit_params make_refit_params(gwnb_geometry_f32 const &g, gwnb_bvh4_f32 const *bvh) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    refit_params p{};
    p.g = g;
    p.nodes = reinterpret_cast<node4 *>(bvh->nodes);
    p.node_count = bvh->node_count;
    p.primitive_indices = bvh->primitive_indices;
    p.triangles = reinterpret_cast<triangle *>(bvh->triangles);
    p.tri48 = a->tri48;
    p.primitive_count = bvh->primitive_count;
    p.parent_slot = a->parent_slot;
    p.expected = a->expected;
    p.arrivals = a->arrivals;
    p.leaf_nodes = a->leaf_nodes;
    p.leaf_node_count = a->leaf_node_count;
    p.root_bounds = a->root_bounds;
    p.status = a->status;
    return p;
}

moment_params make_moment_params(gwnb_bvh4_f32 const *bvh, gwnb_moment4_f32 const *m) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    auto *ma = reinterpret_cast<moment_aux_impl *>(m->aux);
    moment_params p{};
    p.nodes = reinterpret_cast<node4 const *>(bvh->nodes);
    p.node_count = bvh->node_count;
    p.triangles = reinterpret_cast<triangle const *>(bvh->triangles);
    p.primitive_count = bvh->primitive_count;
    p.parent_slot = a->parent_slot;
    p.expected = a->expected;
    p.arrivals = a->arrivals + bvh->node_count;
    p.leaf_nodes = a->leaf_nodes;
    p.leaf_node_count = a->leaf_node_count;
    p.ref_nodes = static_cast<float *>(m->nodes);
    p.qnodes = ma->qnodes;
    p.qcounts = ma->qcounts;
    p.pending = ma->payload;
    p.status = a->status;
    return p;
}
} // namespace

int batch_refit_prepare(gwnb_geometry_f32 const *geoms, gwnb_bvh4_f32 *const *bvhs, gwnb_moment4_f32 *const *moms,
                        std::uint32_t n, int order, batch_refit_state *st, cudaStream_t s) {
    std::vector<batch_bounds_mesh> bd(n);
    std::vector<moment_params> md(n);
    std::vector<std::uint64_t> bb(n + 1, 0), mb(n + 1, 0);
    for (std::uint32_t i = 0; i < n; ++i) {
        gwnb_bvh4_f32 const *b = bvhs[i];
        auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
        bd[i].p = make_refit_params(geoms[i], b);
        bool const leaf_root = ref_leaf(b->root.reference);
        bd[i].leaf_root_first = leaf_root ? ref_offset(b->root.reference) : 0;
        bd[i].leaf_root_count = leaf_root ? ref_count(b->root.reference) : 0;
        bb[i + 1] = bb[i] + (leaf_root ? 1 : a->leaf_node_count);
        // a leaf root has no moment nodes (and no moment refit work)
        md[i] = leaf_root ? moment_params{} : make_moment_params(b, moms[i]);
        mb[i + 1] = mb[i] + (leaf_root ? 0 : a->leaf_node_count);
    }
    st->mesh_count = n;
    st->order = order;
    st->bounds_items = bb[n];
    st->moment_items = mb[n];
    // each buffer joins the state as soon as it exists, so batch_refit_release frees it on any
    // failure after this point
    batch_bounds_mesh *dbd = nullptr;
    moment_params *dmd = nullptr;
    GWNB_TRY(alloc(&dbd, n, s));
    st->bounds_meshes = dbd;
    GWNB_TRY(alloc(&dmd, n, s));
    st->moment_meshes = dmd;
    GWNB_TRY(alloc(&st->bounds_begin, n + 1, s));
    GWNB_TRY(alloc(&st->moment_begin, n + 1, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(dbd, bd.data(), n * sizeof(batch_bounds_mesh), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(dmd, md.data(), n * sizeof(moment_params), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(st->bounds_begin, bb.data(), (n + 1) * sizeof(std::uint64_t), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(st->moment_begin, mb.data(), (n + 1) * sizeof(std::uint64_t), cudaMemcpyHostToDevice, s));
    // the host vectors are released on return: wait for the copies
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    return GWNB_OK;
}

int batch_refit_launch(batch_refit_state const &st, int block, bool bounds, bool moments, cudaStream_t s) {
    if (block < 32 || block > k_batch_block_max || (block % 32) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Batch refit block size must be a multiple of 32 in [32, 256].");
    int const sms = device_sm_count();
    auto grid = [&](std::uint64_t items) {
        std::uint64_t const need = (items + block - 1) / block;
        std::uint64_t const cap = static_cast<std::uint64_t>(sms) * (2048 / block);
        return static_cast<unsigned>(need < cap ? need : cap);
    };
    if (bounds && st.bounds_items > 0)
        note_launch(), k_batch_refit_bounds<<<grid(st.bounds_items), block, 0, s>>>(
            static_cast<batch_bounds_mesh const *>(st.bounds_meshes), st.bounds_begin, st.mesh_count);
    if (moments && st.moment_items > 0) {
        auto const *md = static_cast<moment_params const *>(st.moment_meshes);
        unsigned const g = grid(st.moment_items);
        switch (st.order) {
        case 0: note_launch(), k_batch_refit_moments<0><<<g, block, 0, s>>>(md, st.moment_begin, st.mesh_count); break;
        case 1: note_launch(), k_batch_refit_moments<1><<<g, block, 0, s>>>(md, st.moment_begin, st.mesh_count); break;
        default: note_launch(), k_batch_refit_moments<2><<<g, block, 0, s>>>(md, st.moment_begin, st.mesh_count); break;
        }
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

void batch_refit_release(batch_refit_state &st, cudaStream_t s) {
    auto *bd = static_cast<batch_bounds_mesh *>(st.bounds_meshes);
    auto *md = static_cast<moment_params *>(st.moment_meshes);
    release(bd, s);
    release(md, s);
    release(st.bounds_begin, s);
    release(st.moment_begin, s);
    st.bounds_meshes = nullptr;
    st.moment_meshes = nullptr;
}

int refit_bounds_async(gwnb_geometry_f32 const &g, gwnb_bvh4_f32 *bvh, cudaStream_t s) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    refit_params p{};
    p.g = g;
    p.nodes = reinterpret_cast<node4 *>(bvh->nodes);
    p.node_count = bvh->node_count;
    p.primitive_indices = bvh->primitive_indices;
    p.triangles = reinterpret_cast<triangle *>(bvh->triangles);
    p.tri48 = a->tri48;
    p.primitive_count = bvh->primitive_count;
    p.parent_slot = a->parent_slot;
    p.expected = a->expected;
    p.arrivals = a->arrivals;
    p.leaf_nodes = a->leaf_nodes;
    p.leaf_node_count = a->leaf_node_count;
    p.root_bounds = a->root_bounds;
    p.status = a->status;
    if (bvh->root.reference != 0 && ref_leaf(bvh->root.reference)) {
        note_launch(), k_refit_leaf_root<<<1, 1, 0, s>>>(p, ref_offset(bvh->root.reference), ref_count(bvh->root.reference));
    } else if (a->leaf_node_count > 0) {
        note_launch(), k_refit_bounds<<<grid_for(a->leaf_node_count), k_block, 0, s>>>(p);
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

int refit_moments_async(gwnb_bvh4_f32 const *bvh, gwnb_moment4_f32 *m, cudaStream_t s) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(bvh->aux);
    auto *ma = reinterpret_cast<moment_aux_impl *>(m->aux);
    if (bvh->node_count == 0)
        return GWNB_OK;
    moment_params p{};
    p.nodes = reinterpret_cast<node4 const *>(bvh->nodes);
    p.node_count = bvh->node_count;
    p.triangles = reinterpret_cast<triangle const *>(bvh->triangles);
    p.primitive_count = bvh->primitive_count;
    p.parent_slot = a->parent_slot;
    p.expected = a->expected;
    p.arrivals = a->arrivals + bvh->node_count;
    p.leaf_nodes = a->leaf_nodes;
    p.leaf_node_count = a->leaf_node_count;
    p.ref_nodes = static_cast<float *>(m->nodes);
    p.qnodes = ma->qnodes;
    p.qcounts = ma->qcounts;
    p.pending = ma->payload;
    p.status = a->status;
    unsigned const grid = grid_for(a->leaf_node_count);
    if (grid == 0)
        return set_error(GWNB_INTERNAL_ERROR, "bvh.refit.moment: BVH has no leaf-bearing node.");
    switch (m->order) {
    case 0: note_launch(), k_refit_moments<0><<<grid, k_block, 0, s>>>(p); break;
    case 1: note_launch(), k_refit_moments<1><<<grid, k_block, 0, s>>>(p); break;
    default: note_launch(), k_refit_moments<2><<<grid, k_block, 0, s>>>(p); break;
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

std::size_t moment_payload_bytes(int order) {
    return order == 0 ? sizeof(payload<0>) : (order == 1 ? sizeof(payload<1>) : sizeof(payload<2>));
}

} // namespace gwnb
