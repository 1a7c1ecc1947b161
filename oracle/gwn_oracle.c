/*
 * gwn_oracle.c -- CPU restatement of smallgwn's winding-number path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load it. Nothing in the
 * product path (smallgwn_b200/, include/) calls it.
 *
 * Every function cites the smallgwn file:line it restates (paths relative to that project).
 * Compiled with -ffp-contract=off so float arithmetic is plain IEEE single precision; the
 * topology-deciding arithmetic (Morton quantisation, half areas) therefore matches the CUDA
 * library bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    float min_x, min_y, min_z, max_x, max_y, max_z;
} o_aabb;

typedef struct {
    o_aabb bounds;
    uint64_t reference;
} o_child;

typedef struct {
    o_child c[4];
} o_node4;

typedef struct {
    float v0_x, v0_y, v0_z, e1_x, e1_y, e1_z, e2_x, e2_y, e2_z;
} o_tri;

typedef struct {
    uint32_t li, lk, ri, rk; /* kind 1 = internal, 2 = leaf */
} o_bnode;

#define K_INTERNAL 1u
#define K_LEAF 2u
#define INV32 0xffffffffu
#define OFFSET_MASK ((((uint64_t)1) << 47) - 1)
#define VALID_BIT (((uint64_t)1) << 47)

static inline int ref_valid(uint64_t r) { return (r & VALID_BIT) != 0; }
static inline uint32_t ref_count(uint64_t r) { return (uint32_t)(r >> 48); }
static inline int ref_internal(uint64_t r) { return ref_valid(r) && ref_count(r) == 0; }
static inline int ref_leaf(uint64_t r) { return ref_valid(r) && ref_count(r) != 0; }
static inline uint64_t ref_offset(uint64_t r) { return r & OFFSET_MASK; }
static inline uint64_t make_ref(uint64_t off, uint64_t cnt) { return VALID_BIT | off | (cnt << 48); }

/* std::min / std::max operand order (include/gwn/detail/gwn_bvh_build_common.cuh:90-96). */
static inline float fmin_r(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_r(float a, float b) { return (a < b) ? b : a; }

static o_aabb aabb_union(o_aabb l, o_aabb r) {
    o_aabb u = {fmin_r(l.min_x, r.min_x), fmin_r(l.min_y, r.min_y), fmin_r(l.min_z, r.min_z),
                fmax_r(l.max_x, r.max_x), fmax_r(l.max_y, r.max_y), fmax_r(l.max_z, r.max_z)};
    return u;
}

/* gwn_aabb_half_area, detail/gwn_bvh_build_common.cuh:98-104 (products, then left-to-right sum). */
static float half_area(o_aabb b) {
    float dx = fmax_r(b.max_x - b.min_x, 0.0f);
    float dy = fmax_r(b.max_y - b.min_y, 0.0f);
    float dz = fmax_r(b.max_z - b.min_z, 0.0f);
    float p0 = dx * dy, p1 = dy * dz, p2 = dz * dx;
    float s = p0 + p1;
    return s + p2;
}

/* ---------------------------------------------------------------------------------------------- */
/* Exact winding: tests/reference_cpu.cuh:22-82 (normalise, Van Oosterom-Strackee, zero for a     */
/* vertex hit or a vanishing numerator), summed over every triangle, divided by 4 pi.             */

#define DEFINE_EXACT(T, SUFFIX, SQRT, ATAN2)                                                      \
    static T solid_angle_##SUFFIX(T ax, T ay, T az, T bx, T by, T bz, T cx, T cy, T cz, T qx, T qy, \
                                  T qz) {                                                          \
        T qax = ax - qx, qay = ay - qy, qaz = az - qz;                                            \
        T qbx = bx - qx, qby = by - qy, qbz = bz - qz;                                            \
        T qcx = cx - qx, qcy = cy - qy, qcz = cz - qz;                                            \
        T la = SQRT(qax * qax + qay * qay + qaz * qaz);                                           \
        T lb = SQRT(qbx * qbx + qby * qby + qbz * qbz);                                           \
        T lc = SQRT(qcx * qcx + qcy * qcy + qcz * qcz);                                           \
        if (la == (T)0 || lb == (T)0 || lc == (T)0)                                               \
            return (T)0;                                                                          \
        qax /= la; qay /= la; qaz /= la;                                                          \
        qbx /= lb; qby /= lb; qbz /= lb;                                                          \
        qcx /= lc; qcy /= lc; qcz /= lc;                                                          \
        T ux = qbx - qax, uy = qby - qay, uz = qbz - qaz;                                         \
        T vx = qcx - qax, vy = qcy - qay, vz = qcz - qaz;                                         \
        T crx = uy * vz - uz * vy, cry = uz * vx - ux * vz, crz = ux * vy - uy * vx;              \
        T num = qax * crx + qay * cry + qaz * crz;                                                \
        if (num == (T)0)                                                                          \
            return (T)0;                                                                          \
        T den = (T)1 + (qax * qbx + qay * qby + qaz * qbz) + (qax * qcx + qay * qcy + qaz * qcz) + \
                (qbx * qcx + qby * qcy + qbz * qcz);                                              \
        return (T)2 * ATAN2(num, den);                                                            \
    }                                                                                             \
    void oracle_exact_winding_##SUFFIX(const T *vx, const T *vy, const T *vz, uint64_t nv,         \
                                       const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, \
                                       uint64_t nt, const T *qx, const T *qy, const T *qz, T *out, \
                                       uint64_t nq, int threads) {                                 \
        const T k_pi = (T)3.141592653589793238462643383279502884L;                                 \
        (void)threads;                                                                            \
        _Pragma("omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)")   \
        for (int64_t q = 0; q < (int64_t)nq; ++q) {                                               \
            T sum = (T)0;                                                                         \
            for (uint64_t t = 0; t < nt; ++t) {                                                   \
                uint32_t a = i0[t], b = i1[t], c = i2[t];                                         \
                if (a >= nv || b >= nv || c >= nv)                                                \
                    continue;                                                                     \
                sum += solid_angle_##SUFFIX(vx[a], vy[a], vz[a], vx[b], vy[b], vz[b], vx[c], vy[c], \
                                            vz[c], qx[q], qy[q], qz[q]);                          \
            }                                                                                     \
            out[q] = sum / ((T)4 * k_pi);                                                         \
        }                                                                                         \
    }

DEFINE_EXACT(float, f32, sqrtf, atan2f)
DEFINE_EXACT(double, f64, sqrt, atan2)

/* Exact winding over leaf-ordered triangle records, gwn_winding_number_exact_impl
 * (detail/gwn_query_winding_impl.cuh:377-389): vertices b = v0 + e1, c = v0 + e2. */
static float record_solid_angle(const o_tri *t, float qx, float qy, float qz) {
    return solid_angle_f32(t->v0_x, t->v0_y, t->v0_z, t->v0_x + t->e1_x, t->v0_y + t->e1_y,
                           t->v0_z + t->e1_z, t->v0_x + t->e2_x, t->v0_y + t->e2_y, t->v0_z + t->e2_z,
                           qx, qy, qz);
}

/* ---------------------------------------------------------------------------------------------- */
/* Scene bounds, triangle AABBs and Morton codes: detail/gwn_bvh_build_common.cuh:22-88 (traits,  */
/* clamp, quantise, interleave), :157-214 (per-triangle functor), :243-274 (scene inverse).        */

static uint32_t expand10(uint32_t v) {
    uint32_t x = v & 0x000003ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
static uint64_t expand21(uint64_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}
static float clamp01(float v) {
    if (v < 0.0f)
        return 0.0f;
    if (v > 1.0f)
        return 1.0f;
    return v;
}

/* bits = 32 or 64; codes are written as uint64 either way. scene_out (9 floats) = min, max, inv. */
void oracle_scene_and_morton(const float *vx, const float *vy, const float *vz, uint64_t nv,
                             const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, uint64_t nt,
                             int bits, o_aabb *aabbs, uint64_t *codes, float *scene_out) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t i = 0; i < nv; ++i) {
        float v[3] = {vx[i], vy[i], vz[i]};
        for (int a = 0; a < 3; ++a) {
            mn[a] = fmin_r(mn[a], v[a]);
            mx[a] = fmax_r(mx[a], v[a]);
        }
    }
    float inv[3];
    for (int a = 0; a < 3; ++a)
        inv[a] = (mx[a] == mn[a]) ? 1.0f : 1.0f / (mx[a] - mn[a]);
    if (scene_out) {
        for (int a = 0; a < 3; ++a) {
            scene_out[a] = mn[a];
            scene_out[3 + a] = mx[a];
            scene_out[6 + a] = inv[a];
        }
    }
    for (uint64_t t = 0; t < nt; ++t) {
        uint32_t a = i0[t], b = i1[t], c = i2[t];
        if (a >= nv || b >= nv || c >= nv) {
            memset(&aabbs[t], 0, sizeof(o_aabb));
            codes[t] = 0;
            continue;
        }
        o_aabb bb = {fmin_r(vx[a], fmin_r(vx[b], vx[c])), fmin_r(vy[a], fmin_r(vy[b], vy[c])),
                     fmin_r(vz[a], fmin_r(vz[b], vz[c])), fmax_r(vx[a], fmax_r(vx[b], vx[c])),
                     fmax_r(vy[a], fmax_r(vy[b], vy[c])), fmax_r(vz[a], fmax_r(vz[b], vz[c]))};
        aabbs[t] = bb;
        float ctr[3] = {(bb.min_x + bb.max_x) * 0.5f, (bb.min_y + bb.max_y) * 0.5f,
                        (bb.min_z + bb.max_z) * 0.5f};
        if (bits == 32) {
            uint32_t q[3];
            for (int k = 0; k < 3; ++k)
                q[k] = (uint32_t)(clamp01((ctr[k] - mn[k]) * inv[k]) * 1023.0f);
            codes[t] = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
        } else {
            uint64_t q[3];
            for (int k = 0; k < 3; ++k)
                q[k] = (uint64_t)(clamp01((ctr[k] - mn[k]) * inv[k]) * 2097151.0f);
            codes[t] = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
        }
    }
}

/* Stable sort of (code, id) pairs -- the permutation cub::DeviceRadixSort::SortPairs produces
 * for keys over bits [0, 64) at detail/gwn_bvh_build_common.cuh:332-347. LSD radix, 16-bit digits. */
void oracle_sort_pairs(const uint64_t *codes, uint64_t n, uint64_t *sorted, uint32_t *ids) {
    uint64_t *k0 = (uint64_t *)malloc(n * sizeof(uint64_t)), *k1 = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint32_t *v0 = (uint32_t *)malloc(n * sizeof(uint32_t)), *v1 = (uint32_t *)malloc(n * sizeof(uint32_t));
    uint64_t *cnt = (uint64_t *)malloc(65536 * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) {
        k0[i] = codes[i];
        v0[i] = (uint32_t)i;
    }
    for (int pass = 0; pass < 4; ++pass) {
        int sh = 16 * pass;
        memset(cnt, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; ++i)
            cnt[(k0[i] >> sh) & 0xffffu]++;
        uint64_t acc = 0;
        for (int d = 0; d < 65536; ++d) {
            uint64_t c = cnt[d];
            cnt[d] = acc;
            acc += c;
        }
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t pos = cnt[(k0[i] >> sh) & 0xffffu]++;
            k1[pos] = k0[i];
            v1[pos] = v0[i];
        }
        uint64_t *tk = k0; k0 = k1; k1 = tk;
        uint32_t *tv = v0; v0 = v1; v1 = tv;
    }
    memcpy(sorted, k0, n * sizeof(uint64_t));
    memcpy(ids, v0, n * sizeof(uint32_t));
    free(k0); free(k1); free(v0); free(v1); free(cnt);
}

/* ---------------------------------------------------------------------------------------------- */
/* Karras LBVH: detail/gwn_bvh_build_binary.cuh:29-129 (delta with index tie-break),             */
/* bounds: :131-192 (union of the two children, bottom up).                                        */

static int clz64(uint64_t v) { return v == 0 ? 64 : __builtin_clzll(v); }
static int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

static int k_delta(const uint64_t *codes, int bits, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n)
        return -1;
    uint64_t ci = codes[i], cj = codes[j];
    if (ci == cj) {
        uint64_t diff = (uint64_t)i ^ (uint64_t)j;
        if (diff == 0)
            return bits + 64;
        return bits + clz64(diff);
    }
    if (bits == 32)
        return clz32((uint32_t)(ci ^ cj));
    return clz64(ci ^ cj);
}

/* parents: (parent << 1) | slot for internal nodes (n-1) and leaves (n); INV for the root. */
void oracle_karras(const uint64_t *codes, int bits, uint64_t n, o_bnode *nodes, uint32_t *internal_parent,
                   uint32_t *leaf_parent) {
    for (uint64_t i = 0; i + 1 < n; ++i)
        internal_parent[i] = INV32;
    for (uint64_t i = 0; i < n; ++i)
        leaf_parent[i] = INV32;
    for (int64_t i = 0; i + 1 < (int64_t)n; ++i) {
        int dir = (k_delta(codes, bits, n, i, i + 1) - k_delta(codes, bits, n, i, i - 1) >= 0) ? 1 : -1;
        int dmin = k_delta(codes, bits, n, i, i - dir);
        int64_t lmax = 2;
        while (k_delta(codes, bits, n, i, i + lmax * dir) > dmin)
            lmax <<= 1;
        int64_t l = 0;
        for (int64_t t = lmax >> 1; t > 0; t >>= 1)
            if (k_delta(codes, bits, n, i, i + (l + t) * dir) > dmin)
                l += t;
        int64_t j = i + l * dir;
        int64_t first = i < j ? i : j, last = i < j ? j : i;
        int dnode = k_delta(codes, bits, n, first, last);
        int64_t split = first, step = last - first;
        do {
            step = (step + 1) >> 1;
            int64_t cand = split + step;
            if (cand < last && k_delta(codes, bits, n, first, cand) > dnode)
                split = cand;
        } while (step > 1);
        o_bnode nd;
        nd.li = (uint32_t)split;
        nd.lk = (split == first) ? K_LEAF : K_INTERNAL;
        nd.ri = (uint32_t)(split + 1);
        nd.rk = (split + 1 == last) ? K_LEAF : K_INTERNAL;
        nodes[i] = nd;
        uint32_t me2 = (uint32_t)i << 1;
        if (nd.lk == K_INTERNAL) internal_parent[nd.li] = me2; else leaf_parent[nd.li] = me2;
        if (nd.rk == K_INTERNAL) internal_parent[nd.ri] = me2 | 1u; else leaf_parent[nd.ri] = me2 | 1u;
    }
}

static o_aabb binary_bounds_rec(const o_bnode *nodes, const o_aabb *leaf, o_aabb *out, uint32_t idx,
                                uint32_t kind) {
    if (kind == K_LEAF)
        return leaf[idx];
    /* iterative post-order to avoid deep recursion on degenerate trees */
    (void)nodes; (void)out;
    return leaf[0];
}

/* Bottom-up bounds for any binary hierarchy (children before parents not assumed). */
void oracle_binary_bounds(const o_bnode *nodes, uint64_t n, const o_aabb *leaf, uint32_t root, o_aabb *out) {
    (void)binary_bounds_rec;
    if (n < 2)
        return;
    uint32_t *stack = (uint32_t *)malloc(2 * n * sizeof(uint32_t));
    uint8_t *state = (uint8_t *)calloc(n, 1);
    int64_t sp = 0;
    stack[sp++] = root;
    while (sp > 0) {
        uint32_t v = stack[sp - 1];
        o_bnode nd = nodes[v];
        if (!state[v]) {
            state[v] = 1;
            if (nd.rk == K_INTERNAL) stack[sp++] = nd.ri;
            if (nd.lk == K_INTERNAL) stack[sp++] = nd.li;
            continue;
        }
        --sp;
        o_aabb l = nd.lk == K_LEAF ? leaf[nd.li] : out[nd.li];
        o_aabb r = nd.rk == K_LEAF ? leaf[nd.ri] : out[nd.ri];
        out[v] = aabb_union(l, r);
    }
    free(stack);
    free(state);
}

/* ---------------------------------------------------------------------------------------------- */
/* H-PLOC: detail/gwn_bvh_build_hploc.cuh:104-478, simulated one leaf path at a time. Each range */
/* is merged from the cluster lists of its two halves, so the tree does not depend on the order  */
/* the paths run in; internal ids are assigned sequentially here.                                  */

static uint64_t h_delta(const uint64_t *codes, int bits, uint32_t a, uint32_t b) {
    if (bits == 32) {
        uint64_t ca = (codes[a] << 32) | a, cb = (codes[b] << 32) | b;
        return ca ^ cb;
    }
    uint64_t d = codes[a] ^ codes[b];
    return d == 0 ? (uint64_t)(a ^ b) : d;
}

typedef struct {
    const uint64_t *codes;
    int bits;
    uint32_t n;
    uint32_t radius;
    const o_aabb *leaf;
    o_bnode *nodes;
    o_aabb *ib;
    uint32_t *cluster;
    uint32_t next_id;
    int failed;
} hploc_state;

static uint32_t f_bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static void hploc_merge_range(hploc_state *st, uint32_t left, uint32_t right, uint32_t split, int fin) {
    uint32_t cid[32];
    o_aabb b[32];
    uint32_t r_end = right + 1;
    for (int l = 0; l < 32; ++l)
        cid[l] = INV32;
    /* left list (up to 16) then right list */
    uint32_t nl = 0, nr = 0;
    uint32_t cntl = (split - left) < 16 ? (split - left) : 16;
    for (uint32_t k = 0; k < cntl; ++k)
        cid[k] = st->cluster[left + k];
    for (uint32_t k = 0; k < cntl; ++k)
        nl += cid[k] != INV32;
    uint32_t cntr = (r_end - split) < 16 ? (r_end - split) : 16;
    for (uint32_t k = 0; k < cntr; ++k)
        cid[nl + k] = st->cluster[split + k];
    for (uint32_t k = 0; k < cntr; ++k)
        nr += cid[nl + k] != INV32;
    uint32_t num = nl + nr;
    for (uint32_t l = 0; l < 32; ++l) {
        if (l < num)
            b[l] = cid[l] < st->n ? st->leaf[cid[l]] : st->ib[cid[l] - st->n];
        else
            memset(&b[l], 0, sizeof(o_aabb));
    }
    uint32_t threshold = fin ? 1u : 16u;
    int guard = 0;
    while (num > threshold) {
        uint32_t prev = num;
        /* nearest neighbour with packed keys (:195-241) */
        uint32_t best[32], nk[32], nn[32];
        for (int l = 0; l < 32; ++l)
            best[l] = 0xffffffffu;
        for (uint32_t r = 1; r <= 8 && r <= st->radius; ++r) {
            uint32_t right_key[32];
            int nvalid[32];
            for (uint32_t l = 0; l < 32; ++l) {
                uint32_t nlane = l + r;
                nvalid[l] = nlane < num;
                right_key[l] = 0xffffffffu;
                if (nvalid[l]) {
                    float area = half_area(aabb_union(b[l], b[nlane]));
                    uint32_t akey = (f_bits(area) << 1) & ~0xfu;
                    uint32_t rel = (r - 1u) << 1;
                    right_key[l] = akey | rel | ((nlane & 1u) ^ 1u);
                    uint32_t lk = akey | rel | (l & 1u);
                    if (lk < best[l])
                        best[l] = lk;
                }
            }
            for (uint32_t l = 0; l < 32; ++l) {
                uint32_t src = nvalid[l] ? l + r : l;
                nk[l] = best[src];
                if (nvalid[l] && right_key[l] < nk[l])
                    nk[l] = right_key[l];
            }
            for (uint32_t l = 0; l < 32; ++l)
                if ((int)l - (int)r >= 0)
                    best[l] = nk[l - r];
        }
        for (uint32_t l = 0; l < 32; ++l) {
            uint32_t off = ((best[l] & 0xfu) >> 1) + 1u;
            int rightward = ((best[l] ^ l) & 1u) == 0u;
            nn[l] = rightward ? l + off : l - off;
        }
        /* merge mutual pairs (:300-399) */
        uint32_t safe[32];
        int mutual[32], domerge[32];
        for (uint32_t l = 0; l < 32; ++l) {
            int active = l < num;
            int nv = nn[l] < num && nn[l] != l;
            if (active && !nv)
                st->failed = 1;
            safe[l] = nv ? nn[l] : l;
        }
        uint32_t mcount = 0;
        for (uint32_t l = 0; l < 32; ++l) {
            int active = l < num;
            int nv = nn[l] < num && nn[l] != l;
            mutual[l] = active && nv && l == safe[safe[l]];
            domerge[l] = mutual[l] && l < safe[l];
            mcount += domerge[l];
        }
        uint32_t base = st->next_id;
        st->next_id += mcount;
        uint32_t rel = 0;
        uint32_t ncid[32];
        o_aabb nb[32];
        for (uint32_t l = 0; l < 32; ++l) {
            ncid[l] = cid[safe[l]];
            nb[l] = b[safe[l]];
        }
        for (uint32_t l = 0; l < 32; ++l) {
            if (!domerge[l])
                continue;
            uint32_t merged = base + rel++;
            if (merged < st->n || merged >= 2 * st->n - 1) {
                st->failed = 1;
                continue;
            }
            o_aabb mb = aabb_union(b[l], nb[l]);
            uint32_t iid = merged - st->n;
            o_bnode nd;
            nd.li = cid[l] < st->n ? cid[l] : cid[l] - st->n;
            nd.lk = cid[l] < st->n ? K_LEAF : K_INTERNAL;
            nd.ri = ncid[l] < st->n ? ncid[l] : ncid[l] - st->n;
            nd.rk = ncid[l] < st->n ? K_LEAF : K_INTERNAL;
            st->nodes[iid] = nd;
            st->ib[iid] = mb;
            cid[l] = merged;
            b[l] = mb;
        }
        /* compaction: keep merged lanes and non-mutual lanes, in lane order */
        uint32_t kc[32];
        o_aabb kb[32];
        uint32_t kept = 0;
        for (uint32_t l = 0; l < 32; ++l) {
            if (domerge[l] || !mutual[l]) {
                kc[kept] = cid[l];
                kb[kept] = b[l];
                ++kept;
            }
        }
        for (uint32_t l = 0; l < 32; ++l) {
            if (l < kept) {
                cid[l] = kc[l];
                b[l] = kb[l];
            } else {
                cid[l] = INV32;
            }
        }
        num -= mcount;
        if (num == prev || ++guard > 64) {
            st->failed = 1;
            break;
        }
    }
    for (uint32_t l = 0; l < nl + nr; ++l)
        st->cluster[left + l] = cid[l];
}

/* Returns 0 on success; *root = n - 2. codes are uint64 holding 32- or 64-bit Morton codes. */
int oracle_hploc(const uint64_t *codes, int bits, uint64_t n64, const o_aabb *leaf, uint32_t radius,
                 o_bnode *nodes, o_aabb *ib, uint32_t *root) {
    uint32_t n = (uint32_t)n64;
    *root = INV32;
    if (n < 2)
        return 0;
    hploc_state st = {codes, bits, n, radius, leaf, nodes, ib, NULL, n, 0};
    st.cluster = (uint32_t *)malloc(n * sizeof(uint32_t));
    uint32_t *bp = (uint32_t *)malloc(n * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        st.cluster[i] = i;
        bp[i] = INV32;
    }
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t left = i, right = i, split = 0;
        for (;;) {
            uint32_t prev;
            int is_right = left == 0 ||
                           (right != n - 1 && h_delta(codes, bits, right, right + 1) < h_delta(codes, bits, left - 1, left));
            if (is_right) {
                prev = bp[right];
                bp[right] = left;
                if (prev != INV32) {
                    split = right + 1;
                    right = prev;
                }
            } else {
                prev = bp[left - 1];
                bp[left - 1] = right;
                if (prev != INV32) {
                    split = left;
                    left = prev;
                }
            }
            if (prev == INV32)
                break;
            uint32_t size = right - left + 1;
            int fin = size == n;
            if (size > 16 || fin)
                hploc_merge_range(&st, left, right, split, fin);
        }
    }
    free(st.cluster);
    free(bp);
    if (st.failed || st.next_id != 2 * n - 1)
        return 1;
    *root = n - 2;
    return 0;
}

/* ---------------------------------------------------------------------------------------------- */
/* BVH4 collapse, rule of detail/gwn_bvh_build_collapse.cuh:163-199 (expand the internal candidate */
/* with the largest half area; equal areas keep the lower binary index; the expanded candidate's   */
/* left child takes its slot and the right child is appended). Nodes are numbered breadth first,   */
/* children of a node consecutively in slot order. Stack bounds follow :266-296.                   */

int oracle_collapse(const o_bnode *bin, const o_aabb *bb, const o_aabb *leaf, uint64_t n, uint32_t root,
                    o_node4 *nodes, uint64_t *node_count, uint32_t *internal_bound, uint32_t *packed_bound) {
    if (n < 2) {
        *node_count = 0;
        *internal_bound = 0;
        *packed_bound = 0;
        return 0;
    }
    typedef struct {
        uint32_t b, pi, pp;
    } item;
    item *q = (item *)malloc((n - 1) * sizeof(item));
    uint64_t head = 0, tail = 0;
    q[tail++] = (item){root, 0, 0};
    uint32_t ib_max = 0, pb_max = 0;
    while (head < tail) {
        item it = q[head];
        uint64_t w = head++;
        uint32_t ci[4], ck[4];
        o_bnode r = bin[it.b];
        ci[0] = r.li; ck[0] = r.lk; ci[1] = r.ri; ck[1] = r.rk;
        int k = 2;
        while (k < 4) {
            int best = -1;
            float best_area = -INFINITY;
            uint32_t best_index = INV32;
            for (int c = 0; c < k; ++c) {
                if (ck[c] != K_INTERNAL)
                    continue;
                float area = half_area(bb[ci[c]]);
                if (best >= 0 && area < best_area)
                    continue;
                if (best >= 0 && area == best_area && ci[c] >= best_index)
                    continue;
                best = c;
                best_area = area;
                best_index = ci[c];
            }
            if (best < 0)
                break;
            o_bnode e = bin[ci[best]];
            ci[best] = e.li; ck[best] = e.lk;
            ci[k] = e.ri; ck[k] = e.rk;
            ++k;
        }
        uint32_t kint = 0;
        for (int c = 0; c < k; ++c)
            kint += ck[c] == K_INTERNAL;
        uint32_t nib = it.pi + (kint > 0 ? kint - 1 : 0);
        uint32_t npb = it.pp + (uint32_t)(k - 1);
        if (nib > ib_max) ib_max = nib;
        if (npb > pb_max) pb_max = npb;
        o_node4 nd;
        memset(&nd, 0, sizeof(nd));
        for (int c = 0; c < k; ++c) {
            if (ck[c] == K_LEAF) {
                nd.c[c].bounds = leaf[ci[c]];
                nd.c[c].reference = make_ref(ci[c], 1);
            } else {
                nd.c[c].bounds = bb[ci[c]];
                nd.c[c].reference = make_ref(tail, 0);
                q[tail++] = (item){ci[c], nib, npb};
            }
        }
        nodes[w] = nd;
    }
    *node_count = tail;
    *internal_bound = ib_max;
    *packed_bound = pb_max;
    free(q);
    return 0;
}

/* Leaf-ordered triangle records, detail/gwn_bvh_triangle_impl.cuh:24-67. Returns nonzero on an
 * invalid index. */
int oracle_triangles(const float *vx, const float *vy, const float *vz, uint64_t nv, const uint32_t *i0,
                     const uint32_t *i1, const uint32_t *i2, uint64_t nt, const uint32_t *ids, o_tri *out) {
    int bad = 0;
    for (uint64_t s = 0; s < nt; ++s) {
        uint32_t t = ids[s];
        if (t >= nt) {
            bad = 1;
            continue;
        }
        uint32_t a = i0[t], b = i1[t], c = i2[t];
        if (a >= nv || b >= nv || c >= nv) {
            bad = 1;
            continue;
        }
        o_tri r = {vx[a], vy[a], vz[a], vx[b] - vx[a], vy[b] - vy[a], vz[b] - vz[a],
                   vx[c] - vx[a], vy[c] - vy[a], vz[c] - vz[a]};
        out[s] = r;
    }
    return bad;
}

/* ---------------------------------------------------------------------------------------------- */
/* Taylor moments: detail/gwn_bvh_refit_common.cuh:123-387 (per-triangle raw moments including     */
/* the HDK split integrals for order 2), :67-111 (accumulation), :514-608 (recentring, packing),   */
/* :113-121 (far-field radius). Output: gwn_bvh_moment_node<4, order, float> field-SoA.            */

typedef struct {
    float area, apx, apy, apz, nx, ny, nz;
    float F[3][3];  /* n_i * centroid_j */
    float R[3][6];  /* raw second moments */
} o_payload;

static void pay_acc(o_payload *d, const o_payload *s) {
    d->area += s->area; d->apx += s->apx; d->apy += s->apy; d->apz += s->apz;
    d->nx += s->nx; d->ny += s->ny; d->nz += s->nz;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            d->F[i][j] += s->F[i][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 6; ++j)
            d->R[i][j] += s->R[i][j];
}

static void split_int(float vs[3][3], int va, int vb, int vc, int i, const float P[3], float *oii, float *oij,
                      float *oik) {
    int j = (i == 2) ? 0 : i + 1;
    int k = (j == 2) ? 0 : j + 1;
    float oab_i = vs[vb][i] - vs[va][i], oab_j = vs[vb][j] - vs[va][j], oab_k = vs[vb][k] - vs[va][k];
    float oac_i = vs[vc][i] - vs[va][i], oac_j = vs[vc][j] - vs[va][j], oac_k = vs[vc][k] - vs[va][k];
    float ocb_i = vs[vb][i] - vs[vc][i], ocb_j = vs[vb][j] - vs[vc][j], ocb_k = vs[vb][k] - vs[vc][k];
    float t = (oac_i > 0.0f) ? (oab_i / oac_i) : 0.0f;
    float jd = t * oac_j - oab_j, kd = t * oac_k - oab_k;
    float ca0 = jd * oab_k - kd * oab_j, ca1 = kd * oab_i, ca2 = jd * oab_i;
    float cc0 = jd * ocb_k - kd * ocb_j, cc1 = kd * ocb_i, cc2 = jd * ocb_i;
    float sa = sqrtf(fmax_r(ca0 * ca0 + ca1 * ca1 + ca2 * ca2, 0.0f));
    float sc = sqrtf(fmax_r(cc0 * cc0 + cc1 * cc1 + cc2 * cc2, 0.0f));
    float pai = vs[va][i] - P[i], pci = vs[vc][i] - P[i];
    *oii = sa * (0.5f * pai * pai + (2.0f / 3.0f) * pai * oab_i + 0.25f * oab_i * oab_i) +
           sc * (0.5f * pci * pci + (2.0f / 3.0f) * pci * ocb_i + 0.25f * ocb_i * ocb_i);
    for (int w = 0; w < 2; ++w) {
        float *out = w == 0 ? oij : oik;
        int jk = w == 0 ? j : k;
        float diff = w == 0 ? jd : kd;
        if (!out)
            continue;
        float mid = vs[vb][jk] + 0.5f * diff;
        float amid = mid - vs[va][jk], cmid = mid - vs[vc][jk];
        float paj = vs[va][jk] - P[jk], pcj = vs[vc][jk] - P[jk];
        *out = sa * (0.5f * pai * paj + (1.0f / 3.0f) * pai * amid + (1.0f / 3.0f) * paj * oab_i +
                     0.25f * oab_i * amid) +
               sc * (0.5f * pci * pcj + (1.0f / 3.0f) * pci * cmid + (1.0f / 3.0f) * pcj * ocb_i +
                     0.25f * ocb_i * cmid);
    }
}

static void tri_moment(const o_tri *t, int order, o_payload *m) {
    memset(m, 0, sizeof(*m));
    float ax = t->v0_x, ay = t->v0_y, az = t->v0_z;
    float bx = ax + t->e1_x, by = ay + t->e1_y, bz = az + t->e1_z;
    float cx = ax + t->e2_x, cy = ay + t->e2_y, cz = az + t->e2_z;
    float px = (ax + bx + cx) / 3.0f, py = (ay + by + cy) / 3.0f, pz = (az + bz + cz) / 3.0f;
    float abx = bx - ax, aby = by - ay, abz = bz - az, acx = cx - ax, acy = cy - ay, acz = cz - az;
    float nx = 0.5f * (aby * acz - abz * acy), ny = 0.5f * (abz * acx - abx * acz), nz = 0.5f * (abx * acy - aby * acx);
    float area = sqrtf(fmax_r(nx * nx + ny * ny + nz * nz, 0.0f));
    m->area = area;
    m->apx = px * area; m->apy = py * area; m->apz = pz * area;
    m->nx = nx; m->ny = ny; m->nz = nz;
    float N[3] = {nx, ny, nz}, P[3] = {px, py, pz};
    if (order >= 1)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                m->F[i][j] = N[i] * P[j];
    if (order >= 2 && area != 0.0f) {
        float inv_area = 1.0f / area;
        float nh[3] = {nx * inv_area, ny * inv_area, nz * inv_area};
        float vs[3][3] = {{ax, ay, az}, {bx, by, bz}, {cx, cy, cz}};
        int ord[3][3];
        float span[3];
        for (int a = 0; a < 3; ++a) {
            int o0 = 0, o1 = 1, o2 = 2, tmp;
            if (vs[0][a] > vs[1][a]) { tmp = o0; o0 = o1; o1 = tmp; }
            if (vs[o0][a] > vs[2][a]) { tmp = o0; o0 = o2; o2 = tmp; }
            if (vs[o1][a] > vs[o2][a]) { tmp = o1; o1 = o2; o2 = tmp; }
            ord[a][0] = o0; ord[a][1] = o1; ord[a][2] = o2;
            span[a] = vs[o2][a] - vs[o0][a];
        }
        float ixx = 0, iyy = 0, izz = 0, ixy = 0, iyz = 0, izx = 0;
        float dx = span[0], dy = span[1], dz = span[2];
        if (dx > 0.0f)
            split_int(vs, ord[0][0], ord[0][1], ord[0][2], 0, P, &ixx, (dx >= dy && dy > 0.0f) ? &ixy : NULL,
                      (dx >= dz && dz > 0.0f) ? &izx : NULL);
        if (dy > 0.0f)
            split_int(vs, ord[1][0], ord[1][1], ord[1][2], 1, P, &iyy, (dy >= dz && dz > 0.0f) ? &iyz : NULL,
                      (dx < dy && dx > 0.0f) ? &ixy : NULL);
        if (dz > 0.0f)
            split_int(vs, ord[2][0], ord[2][1], ord[2][2], 2, P, &izz, (dx < dz && dx > 0.0f) ? &izx : NULL,
                      (dy < dz && dy > 0.0f) ? &iyz : NULL);
        float ig[6] = {ixx, iyy, izz, ixy, iyz, izx};
        float pp[6] = {px * px, py * py, pz * pz, px * py, py * pz, pz * px};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 6; ++j)
                m->R[i][j] = nh[i] * ig[j] + N[i] * pp[j];
    }
}

static void finalize_slot(o_aabb b, const o_payload *m, int order, float *f) {
    float ax, ay, az;
    if (m->area > 0.0f) {
        ax = m->apx / m->area; ay = m->apy / m->area; az = m->apz / m->area;
    } else {
        ax = (b.min_x + b.max_x) * 0.5f; ay = (b.min_y + b.max_y) * 0.5f; az = (b.min_z + b.max_z) * 0.5f;
    }
    float dx = fmax_r(ax - b.min_x, b.max_x - ax), dy = fmax_r(ay - b.min_y, b.max_y - ay),
          dz = fmax_r(az - b.min_z, b.max_z - az);
    f[0] = dx * dx + dy * dy + dz * dz;
    f[1] = ax; f[2] = ay; f[3] = az;
    f[4] = m->nx; f[5] = m->ny; f[6] = m->nz;
    if (order >= 1) {
        float xx = m->F[0][0] - ax * m->nx, yy = m->F[1][1] - ay * m->ny, zz = m->F[2][2] - az * m->nz;
        float xy = m->F[0][1] - ay * m->nx, yx = m->F[1][0] - ax * m->ny;
        float yz = m->F[1][2] - az * m->ny, zy = m->F[2][1] - ay * m->nz;
        float zx = m->F[2][0] - ax * m->nz, xz = m->F[0][2] - az * m->nx;
        f[7] = xx; f[8] = yy; f[9] = zz; f[10] = xy + yx; f[11] = yz + zy; f[12] = zx + xz;
    }
    if (order >= 2) {
        float P[3] = {ax, ay, az}, N[3] = {m->nx, m->ny, m->nz};
        float c[3][6];
        for (int i = 0; i < 3; ++i) {
            c[i][0] = m->R[i][0] - 2.0f * P[0] * m->F[i][0] + P[0] * P[0] * N[i];
            c[i][1] = m->R[i][1] - 2.0f * P[1] * m->F[i][1] + P[1] * P[1] * N[i];
            c[i][2] = m->R[i][2] - 2.0f * P[2] * m->F[i][2] + P[2] * P[2] * N[i];
            c[i][3] = m->R[i][3] - P[0] * m->F[i][1] - P[1] * m->F[i][0] + P[0] * P[1] * N[i];
            c[i][4] = m->R[i][4] - P[1] * m->F[i][2] - P[2] * m->F[i][1] + P[1] * P[2] * N[i];
            c[i][5] = m->R[i][5] - P[2] * m->F[i][0] - P[0] * m->F[i][2] + P[2] * P[0] * N[i];
        }
        f[13] = c[0][0]; f[14] = c[1][1]; f[15] = c[2][2];
        f[16] = 2.0f * (c[0][4] + c[1][5] + c[2][3]);
        f[17] = 2.0f * c[0][3] + c[1][0];
        f[18] = 2.0f * c[0][5] + c[2][0];
        f[19] = 2.0f * c[1][4] + c[2][1];
        f[20] = 2.0f * c[1][3] + c[0][1];
        f[21] = 2.0f * c[2][5] + c[0][2];
        f[22] = 2.0f * c[2][4] + c[1][2];
    }
}

static int field_count(int order) { return order == 0 ? 7 : (order == 1 ? 13 : 23); }

/* out: nn * field_count(order) * 4 floats. Children must have larger indices than parents. */
void oracle_moments(int order, const o_node4 *nodes, uint64_t nn, const o_tri *tris, uint64_t nt, float *out) {
    int F = field_count(order);
    o_payload *pend = (o_payload *)calloc(nn ? nn : 1, sizeof(o_payload));
    for (int64_t n = (int64_t)nn - 1; n >= 0; --n) {
        o_payload total;
        memset(&total, 0, sizeof(total));
        int init = 0;
        float *ref = out + (uint64_t)n * F * 4;
        for (int s = 0; s < 4; ++s) {
            uint64_t r = nodes[n].c[s].reference;
            if (!ref_valid(r)) {
                for (int f = 0; f < F; ++f)
                    ref[f * 4 + s] = 0.0f;
                continue;
            }
            o_payload m;
            memset(&m, 0, sizeof(m));
            if (ref_internal(r)) {
                m = pend[ref_offset(r)];
            } else {
                uint64_t first = ref_offset(r);
                uint32_t cnt = ref_count(r);
                for (uint32_t k = 0; k < cnt && first + k < nt; ++k) {
                    o_payload tm;
                    tri_moment(&tris[first + k], order, &tm);
                    if (k == 0) m = tm; else pay_acc(&m, &tm);
                }
            }
            float f[23];
            finalize_slot(nodes[n].c[s].bounds, &m, order, f);
            for (int q = 0; q < F; ++q)
                ref[q * 4 + s] = f[q];
            if (init) pay_acc(&total, &m); else total = m;
            init = 1;
        }
        pend[n] = total;
    }
    free(pend);
}

/* ---------------------------------------------------------------------------------------------- */
/* |q - P|^2 of the acceptance test in one fixed rounding pattern: rx * rx rounded, then two fused  */
/* multiply-adds. The CUDA traversals write the same pattern with __fmul_rn / __fmaf_rn, so the     */
/* oracle's accept / descend decisions equal theirs for the same tree, moments and query.          */
static float accept_dist2(float rx, float ry, float rz) { return fmaf(rz, rz, fmaf(ry, ry, rx * rx)); }

/* ---------------------------------------------------------------------------------------------- */
/* Taylor traversal: gwn_winding_taylor_impl (detail/gwn_query_winding_impl.cuh:101-374), with    */
/* per-query counts of nodes entered, accepted far-field children and exact triangles.             */

static float taylor_one(int order, const o_node4 *nodes, uint64_t nn, const float *mom, const o_tri *tris,
                        uint64_t nt, uint64_t root_ref, float qx, float qy, float qz, float beta2, int cap,
                        uint32_t *st_nodes, uint32_t *st_far, uint32_t *st_near) {
    const float k_pi = 3.14159265358979323846f;
    int F = field_count(order);
    float omega = 0.0f;
    uint32_t sn = 0, sf = 0, snear = 0;
    uint32_t stack[256];
    int sp = 0;
    if (cap > 256) cap = 256;
    if (ref_leaf(root_ref)) {
        uint64_t first = ref_offset(root_ref);
        for (uint32_t k = 0; k < ref_count(root_ref) && first + k < nt; ++k) {
            omega += record_solid_angle(&tris[first + k], qx, qy, qz);
            ++snear;
        }
    } else {
        uint32_t node = (uint32_t)ref_offset(root_ref);
        for (;;) {
            if (node >= nn)
                break;
            ++sn;
            const float *T = mom + (uint64_t)node * F * 4;
            uint32_t next = INV32;
            for (int s = 0; s < 4; ++s) {
                uint64_t r = nodes[node].c[s].reference;
                if (!ref_valid(r))
                    continue;
                float rx = qx - T[1 * 4 + s], ry = qy - T[2 * 4 + s], rz = qz - T[3 * 4 + s];
                float q2 = accept_dist2(rx, ry, rz);
                int descend = !(q2 > 0.0f);
                if (!descend)
                    descend = q2 <= T[0 * 4 + s] * beta2;
                if (!descend) {
                    float m1 = 1.0f / sqrtf(q2);
                    float m2 = m1 * m1, m3 = m2 * m1;
                    float nx = rx * m1, ny = ry * m1, nz = rz * m1;
                    float Nx = T[4 * 4 + s], Ny = T[5 * 4 + s], Nz = T[6 * 4 + s];
                    float rdn = nx * Nx + ny * Ny + nz * Nz;
                    float w = -m2 * rdn;
                    if (order >= 1) {
                        float xx = T[7 * 4 + s], yy = T[8 * 4 + s], zz = T[9 * 4 + s];
                        float xy = T[10 * 4 + s], yz = T[11 * 4 + s], zx = T[12 * 4 + s];
                        float Tt = xx + yy + zz;
                        float S = nx * nx * xx + ny * ny * yy + nz * nz * zz + nx * ny * xy + nx * nz * zx + ny * nz * yz;
                        w += m3 * (Tt - 3.0f * S);
                    }
                    if (order >= 2) {
                        float m4 = m2 * m2;
                        float nx2 = nx * nx, ny2 = ny * ny, nz2 = nz * nz;
                        float nx3 = nx2 * nx, ny3 = ny2 * ny, nz3 = nz2 * nz;
                        float xxx = T[13 * 4 + s], yyy = T[14 * 4 + s], zzz = T[15 * 4 + s], spn = T[16 * 4 + s];
                        float Axy = T[17 * 4 + s], Axz = T[18 * 4 + s], Ayz = T[19 * 4 + s];
                        float Ayx = T[20 * 4 + s], Azx = T[21 * 4 + s], Azy = T[22 * 4 + s];
                        float t0x = Ayx + Azx, t0y = Azy + Axy, t0z = Axz + Ayz;
                        float t1x = ny * Axy + nz * Axz, t1y = nz * Ayz + nx * Ayx, t1z = nx * Azx + ny * Azy;
                        w += m4 * (1.5f * (nx * (3.0f * xxx + t0x) + ny * (3.0f * yyy + t0y) + nz * (3.0f * zzz + t0z)) -
                                   7.5f * (nx3 * xxx + ny3 * yyy + nz3 * zzz + nx * ny * nz * spn + nx2 * t1x +
                                           ny2 * t1y + nz2 * t1z));
                    }
                    if (isfinite(w)) {
                        omega += w;
                        ++sf;
                        continue;
                    }
                }
                if (ref_internal(r)) {
                    if (next != INV32) {
                        if (sp >= cap)
                            return NAN;
                        stack[sp++] = next;
                    }
                    next = (uint32_t)ref_offset(r);
                    continue;
                }
                uint64_t first = ref_offset(r);
                for (uint32_t k = 0; k < ref_count(r) && first + k < nt; ++k) {
                    omega += record_solid_angle(&tris[first + k], qx, qy, qz);
                    ++snear;
                }
            }
            if (next != INV32) {
                node = next;
                continue;
            }
            if (sp == 0)
                break;
            node = stack[--sp];
        }
    }
    if (st_nodes) { *st_nodes = sn; *st_far = sf; *st_near = snear; }
    return omega / (4.0f * k_pi);
}

void oracle_taylor(int order, const o_node4 *nodes, uint64_t nn, const float *mom, const o_tri *tris, uint64_t nt,
                   uint64_t root_ref, const float *qx, const float *qy, const float *qz, uint64_t nq, float beta,
                   int stack_capacity, float *out, uint32_t *stats, int threads) {
    float beta2 = beta * beta;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        uint32_t *st = stats ? stats + 3 * q : NULL;
        out[q] = taylor_one(order, nodes, nn, mom, tris, nt, root_ref, qx[q], qy[q], qz[q], beta2, stack_capacity,
                            st, st ? st + 1 : NULL, st ? st + 2 : NULL);
    }
}

/* Exact winding from leaf-ordered records (linear scan), for parity with the exact batch. */
void oracle_exact_records(const o_tri *tris, uint64_t nt, const float *qx, const float *qy, const float *qz,
                          uint64_t nq, float *out, int threads) {
    const float k_pi = 3.14159265358979323846f;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        float s = 0.0f;
        for (uint64_t t = 0; t < nt; ++t)
            s += record_solid_angle(&tris[t], qx[q], qy[q], qz[q]);
        out[q] = s / (4.0f * k_pi);
    }
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------------------------------------- */
/* Unsigned point-to-mesh distance (brute force, FP64): the closest point on each triangle by the  */
/* Voronoi-region tests of Ericson, Real-Time Collision Detection (2005), section 5.1.5. Used by   */
/* the adjoint checks to keep central-difference stencils away from the surface, where the winding */
/* number jumps.                                                                                  */

static double point_triangle_dist2(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ab[3], ac[3], ap[3], bp[3], cp[3], q[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        ac[k] = c[k] - a[k];
        ap[k] = p[k] - a[k];
        bp[k] = p[k] - b[k];
        cp[k] = p[k] - c[k];
    }
#define DOT3(u, v) ((u)[0] * (v)[0] + (u)[1] * (v)[1] + (u)[2] * (v)[2])
    double d1 = DOT3(ab, ap), d2 = DOT3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0)
        return DOT3(ap, ap);
    double d3 = DOT3(ab, bp), d4 = DOT3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3)
        return DOT3(bp, bp);
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        double v = d1 / (d1 - d3);
        for (int k = 0; k < 3; ++k)
            q[k] = p[k] - (a[k] + v * ab[k]);
        return DOT3(q, q);
    }
    double d5 = DOT3(ab, cp), d6 = DOT3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6)
        return DOT3(cp, cp);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double w = d2 / (d2 - d6);
        for (int k = 0; k < 3; ++k)
            q[k] = p[k] - (a[k] + w * ac[k]);
        return DOT3(q, q);
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; ++k)
            q[k] = p[k] - (b[k] + w * (c[k] - b[k]));
        return DOT3(q, q);
    }
    double den = va + vb + vc;
    if (!(den != 0.0)) /* degenerate triangle: nearest of its vertices */
        return fmin(DOT3(ap, ap), fmin(DOT3(bp, bp), DOT3(cp, cp)));
    double v = vb / den, w = vc / den;
    for (int k = 0; k < 3; ++k)
        q[k] = p[k] - (a[k] + ab[k] * v + ac[k] * w);
    return DOT3(q, q);
#undef DOT3
}

void oracle_mesh_distance_f64(const double *vx, const double *vy, const double *vz, uint64_t nv, const uint32_t *i0,
                              const uint32_t *i1, const uint32_t *i2, uint64_t nt, const double *qx, const double *qy,
                              const double *qz, uint64_t nq, double *out, int threads) {
    (void)threads;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        double p[3] = {qx[q], qy[q], qz[q]};
        double best = INFINITY;
        for (uint64_t t = 0; t < nt; ++t) {
            uint32_t ia = i0[t], ib = i1[t], ic = i2[t];
            if (ia >= nv || ib >= nv || ic >= nv)
                continue;
            double a[3] = {vx[ia], vy[ia], vz[ia]}, b[3] = {vx[ib], vy[ib], vz[ib]}, c[3] = {vx[ic], vy[ic], vz[ic]};
            double d2 = point_triangle_dist2(p, a, b, c);
            if (d2 < best)
                best = d2;
        }
        out[q] = sqrt(best);
    }
}

/* ---------------------------------------------------------------------------------------------- */
/* FP64 Taylor winding numbers (orders 0 and 1) with frozen acceptance decisions: the checker of   */
/* the adjoint. The decisions are those of the float traversal of taylor_one (the test of          */
/* detail/gwn_query_winding_impl.cuh:168-240 on the float moment nodes at the float decision       */
/* point); the sum is then evaluated in FP64 at an FP64 evaluation point, with every slot's         */
/* moments recomputed in FP64 from FP64 vertex positions by the formulas of                         */
/* detail/gwn_bvh_refit_common.cuh:67-121 (N = sum n, P = sum A c / sum A or the box centre,        */
/* M_ij = sum n_i c_j - N_i P_j) and triangles reached in the near field evaluated exactly.          */
/* Central differences of this piecewise-smooth function are what the adjoint must reproduce.      */

typedef struct {
    double area, ac[3], n[3], nc[3][3];
} o_pay64;

typedef struct {
    double P[3], N[3], M[3][3];
} o_slot64;

static void tri_pay64(const double *vx, const double *vy, const double *vz, uint32_t a, uint32_t b, uint32_t c,
                      o_pay64 *m) {
    double v0[3] = {vx[a], vy[a], vz[a]}, v1[3] = {vx[b], vy[b], vz[b]}, v2[3] = {vx[c], vy[c], vz[c]};
    double e1[3], e2[3], ce[3], n[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = v1[k] - v0[k];
        e2[k] = v2[k] - v0[k];
        ce[k] = (v0[k] + v1[k] + v2[k]) / 3.0;
    }
    n[0] = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]);
    n[1] = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]);
    n[2] = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
    m->area = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int i = 0; i < 3; ++i) {
        m->ac[i] = m->area * ce[i];
        m->n[i] = n[i];
        for (int j = 0; j < 3; ++j)
            m->nc[i][j] = n[i] * ce[j];
    }
}

static void pay64_acc(o_pay64 *d, const o_pay64 *s) {
    d->area += s->area;
    for (int i = 0; i < 3; ++i) {
        d->ac[i] += s->ac[i];
        d->n[i] += s->n[i];
        for (int j = 0; j < 3; ++j)
            d->nc[i][j] += s->nc[i][j];
    }
}

static double solid_angle_d(const double a[3], const double b[3], const double c[3]) {
    double la = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double lb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double lc = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (la == 0.0 || lb == 0.0 || lc == 0.0)
        return 0.0;
    double num = a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
                 a[2] * (b[0] * c[1] - b[1] * c[0]);
    if (num == 0.0)
        return 0.0;
    double den = la * lb * lc + (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) * lc +
                 (a[0] * c[0] + a[1] * c[1] + a[2] * c[2]) * lb + (b[0] * c[0] + b[1] * c[1] + b[2] * c[2]) * la;
    return 2.0 * atan2(num, den);
}

/* nodes: the BVH4 (children after parents); mom: the float moment nodes the decisions use;
 * vx/vy/vz: FP64 vertex positions; i0/i1/i2: geometry triangles; prim: sorted -> geometry triangle;
 * d*: float decision points; e*: FP64 evaluation points. out: winding numbers (FP64). */
void oracle_taylor_frozen_f64(int order, const o_node4 *nodes, uint64_t nn, uint64_t root_ref, const float *mom,
                              const double *vx, const double *vy, const double *vz, const uint32_t *i0,
                              const uint32_t *i1, const uint32_t *i2, const uint32_t *prim, uint64_t nt,
                              const float *dx, const float *dy, const float *dz, const double *ex, const double *ey,
                              const double *ez, uint64_t nq, float beta, double *out, int threads) {
    const double k_pi = 3.141592653589793238462643383279502884;
    int F = field_count(order);
    float beta2 = beta * beta;
    o_slot64 *slots = (o_slot64 *)calloc(nn ? nn * 4 : 1, sizeof(o_slot64));
    o_pay64 *pend = (o_pay64 *)calloc(nn ? nn : 1, sizeof(o_pay64));
    for (int64_t n = (int64_t)nn - 1; n >= 0; --n) {
        o_pay64 total;
        memset(&total, 0, sizeof(total));
        for (int s = 0; s < 4; ++s) {
            uint64_t r = nodes[n].c[s].reference;
            if (!ref_valid(r))
                continue;
            o_pay64 m;
            memset(&m, 0, sizeof(m));
            if (ref_internal(r)) {
                m = pend[ref_offset(r)];
            } else {
                for (uint32_t k = 0; k < ref_count(r) && ref_offset(r) + k < nt; ++k) {
                    uint32_t t = prim[ref_offset(r) + k];
                    o_pay64 tm;
                    tri_pay64(vx, vy, vz, i0[t], i1[t], i2[t], &tm);
                    pay64_acc(&m, &tm);
                }
            }
            o_slot64 *sl = &slots[(uint64_t)n * 4 + s];
            o_aabb b = nodes[n].c[s].bounds;
            double P[3];
            if (m.area > 0.0) {
                for (int i = 0; i < 3; ++i)
                    P[i] = m.ac[i] / m.area;
            } else {
                P[0] = 0.5 * ((double)b.min_x + b.max_x);
                P[1] = 0.5 * ((double)b.min_y + b.max_y);
                P[2] = 0.5 * ((double)b.min_z + b.max_z);
            }
            for (int i = 0; i < 3; ++i) {
                sl->P[i] = P[i];
                sl->N[i] = m.n[i];
                for (int j = 0; j < 3; ++j)
                    sl->M[i][j] = m.nc[i][j] - m.n[i] * P[j];
            }
            pay64_acc(&total, &m);
        }
        pend[n] = total;
    }
    (void)threads;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        double e[3] = {ex[q], ey[q], ez[q]};
        double omega = 0.0;
        uint32_t stack[256];
        int sp = 0;
        if (ref_leaf(root_ref)) {
            for (uint32_t k = 0; k < ref_count(root_ref) && ref_offset(root_ref) + k < nt; ++k) {
                uint32_t t = prim[ref_offset(root_ref) + k];
                double a[3] = {vx[i0[t]] - e[0], vy[i0[t]] - e[1], vz[i0[t]] - e[2]};
                double b[3] = {vx[i1[t]] - e[0], vy[i1[t]] - e[1], vz[i1[t]] - e[2]};
                double c[3] = {vx[i2[t]] - e[0], vy[i2[t]] - e[1], vz[i2[t]] - e[2]};
                omega += solid_angle_d(a, b, c);
            }
        } else {
            uint32_t node = (uint32_t)ref_offset(root_ref);
            for (;;) {
                if (node >= nn)
                    break;
                const float *T = mom + (uint64_t)node * F * 4;
                uint32_t next = INV32;
                for (int s = 0; s < 4; ++s) {
                    uint64_t r = nodes[node].c[s].reference;
                    if (!ref_valid(r))
                        continue;
                    float rx = dx[q] - T[1 * 4 + s], ry = dy[q] - T[2 * 4 + s], rz = dz[q] - T[3 * 4 + s];
                    float q2 = accept_dist2(rx, ry, rz);
                    int descend = !(q2 > 0.0f);
                    if (!descend)
                        descend = q2 <= T[0 * 4 + s] * beta2;
                    if (!descend) {
                        const o_slot64 *sl = &slots[(uint64_t)node * 4 + s];
                        double d[3] = {e[0] - sl->P[0], e[1] - sl->P[1], e[2] - sl->P[2]};
                        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        double m1 = 1.0 / sqrt(r2), m2 = m1 * m1, m3 = m2 * m1;
                        double u[3] = {d[0] * m1, d[1] * m1, d[2] * m1};
                        double w = -m2 * (u[0] * sl->N[0] + u[1] * sl->N[1] + u[2] * sl->N[2]);
                        if (order >= 1) {
                            double tr = sl->M[0][0] + sl->M[1][1] + sl->M[2][2];
                            double S = 0.0;
                            for (int i = 0; i < 3; ++i)
                                for (int j = 0; j < 3; ++j)
                                    S += u[i] * sl->M[i][j] * u[j];
                            w += m3 * (tr - 3.0 * S);
                        }
                        omega += w;
                        continue;
                    }
                    if (ref_internal(r)) {
                        if (next != INV32) {
                            if (sp >= 256) {
                                omega = NAN;
                                break;
                            }
                            stack[sp++] = next;
                        }
                        next = (uint32_t)ref_offset(r);
                        continue;
                    }
                    for (uint32_t k = 0; k < ref_count(r) && ref_offset(r) + k < nt; ++k) {
                        uint32_t t = prim[ref_offset(r) + k];
                        double a[3] = {vx[i0[t]] - e[0], vy[i0[t]] - e[1], vz[i0[t]] - e[2]};
                        double b[3] = {vx[i1[t]] - e[0], vy[i1[t]] - e[1], vz[i1[t]] - e[2]};
                        double c[3] = {vx[i2[t]] - e[0], vy[i2[t]] - e[1], vz[i2[t]] - e[2]};
                        omega += solid_angle_d(a, b, c);
                    }
                }
                if (next != INV32) {
                    node = next;
                    continue;
                }
                if (sp == 0)
                    break;
                node = stack[--sp];
            }
        }
        out[q] = omega / (4.0 * k_pi);
    }
    free(slots);
    free(pend);
}

/* ---------------------------------------------------------------------------------------------- */
/* Spatial queries on the BVH4: unsigned point-to-mesh distance and ray first hit.                 */
/* smallgwn's formulas and its canonical near-first traversal (detail/gwn_query_distance_impl.cuh, */
/* detail/gwn_query_ray_impl.cuh), with every dot product, cross product, multiply-add and slab    */
/* bound fused in one fixed pattern (fmaf) that the CUDA kernels use identically; smallgwn leaves   */
/* that contraction to its compiler.                                                             */

#include <float.h>

typedef struct {
    float x, y, z;
} o_v3;

static inline o_v3 v3(float x, float y, float z) {
    o_v3 r = {x, y, z};
    return r;
}
static inline o_v3 v3_add(o_v3 a, o_v3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline o_v3 v3_sub(o_v3 a, o_v3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
/* a * s + c, fused per component */
static inline o_v3 v3_fma(o_v3 a, float s, o_v3 c) { return v3(fmaf(a.x, s, c.x), fmaf(a.y, s, c.y), fmaf(a.z, s, c.z)); }
/* detail/gwn_query_vec3_impl.cuh:109-121, fused: x*x' first, then y and z accumulated */
static inline float v3_dot(o_v3 a, o_v3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
static inline o_v3 v3_cross(o_v3 a, o_v3 b) {
    return v3(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
/* a * b - c * d with the second product rounded first */
static inline float o_dop(float a, float b, float c, float d) { return fmaf(a, b, -(c * d)); }

/* Vertices of a leaf-ordered record, reconstructed as v0 + e (detail/gwn_query_distance_impl.cuh:20-33). */
static inline void record_vertices(const o_tri *t, o_v3 *a, o_v3 *b, o_v3 *c) {
    *a = v3(t->v0_x, t->v0_y, t->v0_z);
    *b = v3(t->v0_x + t->e1_x, t->v0_y + t->e1_y, t->v0_z + t->e1_z);
    *c = v3(t->v0_x + t->e2_x, t->v0_y + t->e2_y, t->v0_z + t->e2_z);
}

/* Squared point-triangle distance, Voronoi-region tests (detail/gwn_query_geometry_impl.cuh:49-100). */
static float o_point_tri_d2(o_v3 p, o_v3 a, o_v3 b, o_v3 c) {
    o_v3 const ab = v3_sub(b, a), ac = v3_sub(c, a), ap = v3_sub(p, a);
    float const d1 = v3_dot(ab, ap), d2 = v3_dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f)
        return v3_dot(ap, ap);
    o_v3 const bp = v3_sub(p, b);
    float const d3 = v3_dot(ab, bp), d4 = v3_dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3)
        return v3_dot(bp, bp);
    float const vc = o_dop(d1, d4, d3, d2);
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float const v = d1 / (d1 - d3);
        o_v3 const q = v3_sub(p, v3_fma(ab, v, a));
        return v3_dot(q, q);
    }
    o_v3 const cp = v3_sub(p, c);
    float const d5 = v3_dot(ab, cp), d6 = v3_dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6)
        return v3_dot(cp, cp);
    float const vb = o_dop(d5, d2, d1, d6);
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float const w = d2 / (d2 - d6);
        o_v3 const q = v3_sub(p, v3_fma(ac, w, a));
        return v3_dot(q, q);
    }
    float const va = o_dop(d3, d6, d5, d4);
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float const w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        o_v3 const q = v3_sub(p, v3_fma(v3_sub(c, b), w, b));
        return v3_dot(q, q);
    }
    float const denom = 1.0f / (va + vb + vc);
    float const v = vb * denom, w = vc * denom;
    o_v3 const q = v3_sub(p, v3_fma(ac, w, v3_fma(ab, v, a)));
    return v3_dot(q, q);
}

/* std::max(v, 0) with its NaN behaviour (the first operand is returned when unordered). */
static inline float o_pos(float v) { return (v < 0.0f) ? 0.0f : v; }

/* detail/gwn_query_geometry_impl.cuh:104-114 */
static inline float o_aabb_d2(float qx, float qy, float qz, const o_aabb *b) {
    float const dx = o_pos(b->min_x - qx) + o_pos(qx - b->max_x);
    float const dy = o_pos(b->min_y - qy) + o_pos(qy - b->max_y);
    float const dz = o_pos(b->min_z - qz) + o_pos(qz - b->max_z);
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

/* One query of detail/gwn_query_distance_impl.cuh:40-160: near-first descent with the culling band
 * as initial bound, leaf children visited inside their node before internal children are queued,
 * an early return of 0 once a triangle touches the query. Stack overflow returns NaN. */
static float o_distance_one(const o_node4 *nodes, uint64_t nn, const o_tri *tris, uint64_t nt, uint64_t root_ref,
                            float qx, float qy, float qz, float culling_band, int cap, uint32_t *st) {
    o_v3 const p = v3(qx, qy, qz);
    float const band = (culling_band < 0.0f) ? 0.0f : culling_band;
    float best = band * band;
    uint32_t n_nodes = 0, n_tris = 0;
    uint64_t stack[256];
    int sp = 0;
    uint64_t ref = root_ref;
    float result = NAN;
    int done = 0;
#define VISIT_LEAF(R, ALIVE)                                                                        \
    do {                                                                                            \
        for (uint32_t k_ = 0; k_ < ref_count(R); ++k_) {                                            \
            uint64_t const si_ = ref_offset(R) + k_;                                                \
            if (si_ >= nt)                                                                          \
                continue;                                                                           \
            o_v3 a_, b_, c_;                                                                        \
            record_vertices(&tris[si_], &a_, &b_, &c_);                                             \
            float const d2_ = o_point_tri_d2(p, a_, b_, c_);                                        \
            ++n_tris;                                                                               \
            if (d2_ < best)                                                                         \
                best = d2_;                                                                         \
        }                                                                                           \
        ALIVE = best > 0.0f;                                                                        \
    } while (0)
    for (;;) {
        uint64_t next = 0;
        if (ref_leaf(ref)) {
            int alive;
            VISIT_LEAF(ref, alive);
            if (!alive) {
                result = 0.0f;
                done = 1;
                break;
            }
        } else if (ref_internal(ref) && ref_offset(ref) < nn) {
            ++n_nodes;
            const o_node4 *nd = &nodes[ref_offset(ref)];
            float cd[4];
            uint64_t cr[4];
            int cnt = 0;
            for (int s = 0; s < 4; ++s) {
                if (!ref_valid(nd->c[s].reference))
                    continue;
                float const d2 = o_aabb_d2(qx, qy, qz, &nd->c[s].bounds);
                if (d2 >= best)
                    continue;
                cd[cnt] = d2;
                cr[cnt] = nd->c[s].reference;
                ++cnt;
            }
            for (int s = cnt; s < 4; ++s) {
                cd[s] = INFINITY;
                cr[s] = 0;
            }
#define CSWAP(L, R)                                                                                 \
    if (cd[L] > cd[R]) {                                                                            \
        float tf_ = cd[L];                                                                          \
        cd[L] = cd[R];                                                                              \
        cd[R] = tf_;                                                                                \
        uint64_t tr_ = cr[L];                                                                       \
        cr[L] = cr[R];                                                                              \
        cr[R] = tr_;                                                                                \
    }
            CSWAP(0, 1) CSWAP(2, 3) CSWAP(0, 2) CSWAP(1, 3) CSWAP(1, 2)
            int stop = 0;
            for (int s = 0; s < cnt && !stop; ++s) {
                if (ref_leaf(cr[s]) && cd[s] < best) {
                    int alive;
                    VISIT_LEAF(cr[s], alive);
                    if (!alive)
                        stop = 1;
                }
            }
            if (stop) {
                result = 0.0f;
                done = 1;
                break;
            }
            for (int s = cnt - 1; s >= 0; --s) {
                if (!ref_internal(cr[s]) || cd[s] >= best)
                    continue;
                if (next != 0) {
                    if (sp >= cap) {
                        done = 1;
                        break;
                    }
                    stack[sp++] = next;
                }
                next = cr[s];
            }
            if (done)
                break; /* overflow: result stays NaN */
        }
        if (next != 0) {
            ref = next;
            continue;
        }
        if (sp == 0)
            break;
        ref = stack[--sp];
    }
#undef VISIT_LEAF
    if (!done)
        result = sqrtf(best);
    if (st) {
        st[0] = n_nodes;
        st[1] = n_tris;
    }
    return result;
}

void oracle_unsigned_distance(const o_node4 *nodes, uint64_t nn, const o_tri *tris, uint64_t nt, uint64_t root_ref,
                              const float *qx, const float *qy, const float *qz, uint64_t n, float culling_band,
                              int stack_capacity, float *out, uint32_t *stats, int threads) {
    int const cap = stack_capacity > 256 ? 256 : stack_capacity;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        out[i] = o_distance_one(nodes, nn, tris, nt, root_ref, qx[i], qy[i], qz[i], culling_band, cap,
                                stats ? stats + 2 * i : NULL);
}

/* Brute force over every record (same per-triangle arithmetic, no pruning): the minimum squared
 * distance under the band, then its square root. */
void oracle_distance_brute(const o_tri *tris, uint64_t nt, const float *qx, const float *qy, const float *qz,
                           uint64_t n, float culling_band, float *out, int threads) {
    float const band = (culling_band < 0.0f) ? 0.0f : culling_band;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        o_v3 const p = v3(qx[i], qy[i], qz[i]);
        float best = band * band;
        for (uint64_t t = 0; t < nt; ++t) {
            o_v3 a, b, c;
            record_vertices(&tris[t], &a, &b, &c);
            float const d2 = o_point_tri_d2(p, a, b, c);
            if (d2 < best)
                best = d2;
        }
        out[i] = sqrtf(best);
    }
}

/* Ray first-hit record; same layout as gwn::gwn_ray_first_hit_result<float, uint32_t>
 * (include/gwn/gwn_query.cuh:63-96): 32 bytes. status 0 miss, 1 hit, 2 overflow. */
typedef struct {
    float t, u, v, nx, ny, nz;
    uint32_t primitive_id;
    uint8_t status;
    uint8_t pad[3];
} o_hit;

/* detail/gwn_query_ray_impl.cuh:63-81: reciprocal direction, parallel axes flagged; here also
 * -o * inv per axis so that a slab bound is one fused lo * inv - o * inv. */
typedef struct {
    float inv[3], noi[3];
    int zero[3];
} o_raydir;

static o_raydir o_make_raydir(const float o[3], float dx, float dy, float dz) {
    o_raydir r;
    float const d[3] = {dx, dy, dz};
    for (int k = 0; k < 3; ++k) {
        r.zero[k] = d[k] == 0.0f;
        r.inv[k] = r.zero[k] ? 0.0f : 1.0f / d[k];
        r.noi[k] = -(o[k] * r.inv[k]);
    }
    return r;
}

/* detail/gwn_query_ray_impl.cuh:84-139 and :259-271: closed slab test against [t_min, t_max]; a
 * parallel axis is a containment test, the others bound the interval (std::min / std::max operand
 * order, axes folded x, y, z). t_max >= t_min holds for every call (the running best never drops
 * below t_min). */
static int o_ray_box(const float o[3], const o_raydir *rd, const o_aabb *b, float t_min, float t_max, float *t_near_out) {
    float t_near = t_min, t_far = t_max;
    float const lo[3] = {b->min_x, b->min_y, b->min_z};
    float const hi[3] = {b->max_x, b->max_y, b->max_z};
    for (int k = 0; k < 3; ++k) {
        if (rd->zero[k]) {
            if (!(o[k] >= lo[k] && o[k] <= hi[k]))
                return 0;
            continue;
        }
        float const t0 = fmaf(lo[k], rd->inv[k], rd->noi[k]);
        float const t1 = fmaf(hi[k], rd->inv[k], rd->noi[k]);
        t_near = fmax_r(t_near, fmin_r(t0, t1));
        t_far = fmin_r(t_far, fmax_r(t0, t1));
    }
    if (!(t_near <= t_far))
        return 0;
    *t_near_out = t_near;
    return 1;
}

/* detail/gwn_query_ray_impl.cuh:142-171: component-wise stable cross products. */
static o_v3 o_stable_normal(o_v3 a, o_v3 b, o_v3 c) {
    float const abx = a.z * b.y, aby = a.x * b.z, abz = a.y * b.x;
    float const bcx = b.z * c.y, bcy = b.x * c.z, bcz = b.y * c.x;
    o_v3 const cab = v3(fmaf(a.y, b.z, -abx), fmaf(a.z, b.x, -aby), fmaf(a.x, b.y, -abz));
    o_v3 n = v3(fmaf(b.y, c.z, -bcx), fmaf(b.z, c.x, -bcy), fmaf(b.x, c.y, -bcz));
    if (fabsf(abx) < fabsf(bcx))
        n.x = cab.x;
    if (fabsf(aby) < fabsf(bcy))
        n.y = cab.y;
    if (fabsf(abz) < fabsf(bcz))
        n.z = cab.z;
    return n;
}

/* detail/gwn_query_ray_impl.cuh:174-238: oriented Pluecker edge functions. */
static int o_ray_tri(o_v3 o, o_v3 d, o_v3 v0, o_v3 v1, o_v3 v2, float t_min, float t_max, float *t_out,
                     float *u_out, float *v_out, o_v3 *n_out) {
    o_v3 const p0 = v3_sub(v0, o), p1 = v3_sub(v1, o), p2 = v3_sub(v2, o);
    o_v3 const e0 = v3_sub(p2, p0), e1 = v3_sub(p0, p1), e2 = v3_sub(p1, p2);
    float const u = v3_dot(v3_cross(e0, v3_add(p2, p0)), d);
    float const v = v3_dot(v3_cross(e1, v3_add(p0, p1)), d);
    float const w = v3_dot(v3_cross(e2, v3_add(p1, p2)), d);
    float const uvw = u + v + w;
    float const eps = FLT_EPSILON * fabsf(uvw);
    float const mn = fmin_r(u, fmin_r(v, w));
    float const mx = fmax_r(u, fmax_r(v, w));
    if (!(mn >= -eps || mx <= eps))
        return 0;
    o_v3 const ng = o_stable_normal(e0, e1, e2);
    float const den = 2.0f * v3_dot(ng, d);
    if (den == 0.0f)
        return 0;
    float const t = (2.0f * v3_dot(p0, ng)) / den;
    if (!(t_min <= t && t <= t_max))
        return 0;
    if (fabsf(uvw) >= FLT_MIN) {
        float const inv = 1.0f / uvw;
        *u_out = u * inv;
        *v_out = v * inv;
    } else {
        if (uvw == 0.0f)
            return 0;
        *u_out = u / uvw;
        *v_out = v / uvw;
    }
    *t_out = t;
    *n_out = ng;
    return 1;
}

typedef struct {
    float t, u, v;
    o_v3 n;
    uint32_t id;
    int found;
} o_best;

/* A candidate replaces the best hit when it is nearer, or equally near with a lower original
 * primitive id (smallgwn keeps the first one its traversal meets, detail/gwn_query_ray_impl.cuh:
 * 436-437; the id rule makes the result independent of the traversal order). */
static void o_ray_leaf(const o_tri *tris, const uint32_t *prim, uint64_t nt, uint64_t r, o_v3 o, o_v3 d, float t_min,
                       o_best *best, uint32_t *n_tris) {
    for (uint32_t k = 0; k < ref_count(r); ++k) {
        uint64_t const si = ref_offset(r) + k;
        if (si >= nt)
            continue;
        o_v3 a, b, c, n;
        record_vertices(&tris[si], &a, &b, &c);
        float t, u, v;
        ++*n_tris;
        if (!o_ray_tri(o, d, a, b, c, t_min, best->t, &t, &u, &v, &n))
            continue;
        uint32_t const id = prim[si];
        if (best->found && !(t < best->t || (t == best->t && id < best->id)))
            continue;
        best->t = t;
        best->u = u;
        best->v = v;
        best->n = n;
        best->id = id;
        best->found = 1;
    }
}

/* One ray of detail/gwn_query_ray_impl.cuh:376-560 (canonical traversal). */
static o_hit o_ray_one(const o_node4 *nodes, uint64_t nn, const o_tri *tris, const uint32_t *prim, uint64_t nt,
                       uint64_t root_ref, const float org[3], const float dir[3], float t_min, float t_max, int cap,
                       uint32_t *st) {
    o_hit h;
    memset(&h, 0, sizeof(h));
    h.t = -1.0f;
    h.primitive_id = 0xffffffffu;
    uint32_t n_nodes = 0, n_tris = 0;
    float const len2 = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
    if (!(len2 > 0.0f)) {
        if (st)
            st[0] = st[1] = 0;
        return h;
    }
    o_v3 const o = v3(org[0], org[1], org[2]), d = v3(dir[0], dir[1], dir[2]);
    o_raydir const rd = o_make_raydir(org, dir[0], dir[1], dir[2]);
    o_best best;
    memset(&best, 0, sizeof(best));
    best.t = t_max;
    uint64_t stack[256];
    int sp = 0, overflow = 0;
    uint64_t ref = root_ref;
    for (;;) {
        uint64_t next = 0;
        if (ref_leaf(ref)) {
            o_ray_leaf(tris, prim, nt, ref, o, d, t_min, &best, &n_tris);
        } else if (ref_internal(ref) && ref_offset(ref) < nn) {
            ++n_nodes;
            const o_node4 *nd = &nodes[ref_offset(ref)];
            float et[4];
            uint64_t cr[4];
            int cnt = 0;
            for (int s = 0; s < 4; ++s) {
                if (!ref_valid(nd->c[s].reference))
                    continue;
                float tn;
                if (!o_ray_box(org, &rd, &nd->c[s].bounds, t_min, best.t, &tn))
                    continue;
                et[cnt] = tn;
                cr[cnt] = nd->c[s].reference;
                ++cnt;
            }
            for (int s = cnt; s < 4; ++s) {
                et[s] = INFINITY;
                cr[s] = 0;
            }
#define ESWAP(L, R)                                                                                 \
    if (et[L] > et[R]) {                                                                            \
        float tf_ = et[L];                                                                          \
        et[L] = et[R];                                                                              \
        et[R] = tf_;                                                                                \
        uint64_t tr_ = cr[L];                                                                       \
        cr[L] = cr[R];                                                                              \
        cr[R] = tr_;                                                                                \
    }
            ESWAP(0, 1) ESWAP(2, 3) ESWAP(0, 2) ESWAP(1, 3) ESWAP(1, 2)
            for (int s = 0; s < cnt; ++s)
                if (ref_leaf(cr[s]) && et[s] <= best.t)
                    o_ray_leaf(tris, prim, nt, cr[s], o, d, t_min, &best, &n_tris);
            for (int s = cnt - 1; s >= 0; --s) {
                if (!ref_internal(cr[s]) || et[s] > best.t)
                    continue;
                if (next != 0) {
                    if (sp >= cap) {
                        overflow = 1;
                        break;
                    }
                    stack[sp++] = next;
                }
                next = cr[s];
            }
            if (overflow)
                break;
        }
        if (next != 0) {
            ref = next;
            continue;
        }
        if (sp == 0)
            break;
        ref = stack[--sp];
    }
    if (best.found) {
        h.t = best.t;
        h.u = best.u;
        h.v = best.v;
        h.nx = best.n.x;
        h.ny = best.n.y;
        h.nz = best.n.z;
        h.primitive_id = best.id;
        h.status = 1;
    }
    if (overflow)
        h.status = 2;
    if (st) {
        st[0] = n_nodes;
        st[1] = n_tris;
    }
    return h;
}

void oracle_ray_first_hit(const o_node4 *nodes, uint64_t nn, const o_tri *tris, const uint32_t *prim, uint64_t nt,
                          uint64_t root_ref, const float *ox, const float *oy, const float *oz, const float *dx,
                          const float *dy, const float *dz, uint64_t n, float t_min, float t_max, int stack_capacity,
                          o_hit *out, uint32_t *stats, int threads) {
    int const cap = stack_capacity > 256 ? 256 : stack_capacity;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float const o[3] = {ox[i], oy[i], oz[i]}, d[3] = {dx[i], dy[i], dz[i]};
        out[i] = o_ray_one(nodes, nn, tris, prim, nt, root_ref, o, d, t_min, t_max, cap, stats ? stats + 2 * i : NULL);
    }
}

/* Brute force over every record with the same per-triangle test and tie rule. */
void oracle_ray_brute(const o_tri *tris, const uint32_t *prim, uint64_t nt, const float *ox, const float *oy,
                      const float *oz, const float *dx, const float *dy, const float *dz, uint64_t n, float t_min,
                      float t_max, o_hit *out, int threads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        o_hit h;
        memset(&h, 0, sizeof(h));
        h.t = -1.0f;
        h.primitive_id = 0xffffffffu;
        float const len2 = dx[i] * dx[i] + dy[i] * dy[i] + dz[i] * dz[i];
        if (len2 > 0.0f) {
            o_v3 const o = v3(ox[i], oy[i], oz[i]), d = v3(dx[i], dy[i], dz[i]);
            o_best best;
            memset(&best, 0, sizeof(best));
            best.t = t_max;
            uint32_t dummy = 0;
            for (uint64_t t = 0; t < nt; ++t)
                o_ray_leaf(tris, prim, nt, make_ref(t, 1), o, d, t_min, &best, &dummy);
            if (best.found) {
                h.t = best.t;
                h.u = best.u;
                h.v = best.v;
                h.nx = best.n.x;
                h.ny = best.n.y;
                h.nz = best.n.z;
                h.primitive_id = best.id;
                h.status = 1;
            }
        }
        out[i] = h;
    }
}

/* ---------------------------------------------------------------------------------------------- */
/* Boundary chain and antipodal winding numbers (smallgwn detail/gwn_boundary_impl.cuh and         */
/* detail/gwn_query_winding_antipodal_impl.cuh; Martens, Trettner and Bessmeltsev, "The Antipodal */
/* Method", ACM TOG 45(4), 2026). Products and sums fused in the pattern of the spatial queries.   */

typedef struct {
    uint64_t key; /* (lo << 32) | hi */
    int orientation;
} o_edge;

static int edge_cmp(const void *a, const void *b) {
    uint64_t const x = ((const o_edge *)a)->key, y = ((const o_edge *)b)->key;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* detail/gwn_boundary_impl.cuh:34-60 and :127-171: every triangle edge keyed by its (low, high)
 * vertex pair with orientation +1 when it runs low to high, -1 when high to low, 0 when both ends
 * coincide; a key whose orientations sum to s != 0 emits one directed edge (low -> high for s > 0,
 * high -> low otherwise) of multiplicity |s|, rows in ascending (low, high) order. Returns the
 * number of rows; with start == NULL only counts. */
uint64_t oracle_boundary_chain(const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, uint64_t nt, uint32_t *start,
                               uint32_t *end, uint64_t *mult) {
    uint64_t const ne = nt * 3;
    o_edge *e = (o_edge *)malloc((ne ? ne : 1) * sizeof(o_edge));
    for (uint64_t t = 0; t < nt; ++t) {
        uint32_t const v[3] = {i0[t], i1[t], i2[t]};
        for (int k = 0; k < 3; ++k) {
            uint32_t const s = v[k], d = v[(k + 1) % 3];
            uint32_t const lo = s < d ? s : d, hi = s < d ? d : s;
            e[t * 3 + k].key = ((uint64_t)lo << 32) | hi;
            e[t * 3 + k].orientation = s < d ? 1 : (d < s ? -1 : 0);
        }
    }
    /* the order within a key group does not matter for the sum */
    qsort(e, ne, sizeof(o_edge), edge_cmp);
    uint64_t rows = 0;
    for (uint64_t i = 0; i < ne;) {
        uint64_t j = i;
        int64_t sum = 0;
        while (j < ne && e[j].key == e[i].key)
            sum += e[j++].orientation;
        if (sum != 0) {
            if (start) {
                uint32_t const lo = (uint32_t)(e[i].key >> 32), hi = (uint32_t)e[i].key;
                start[rows] = sum > 0 ? lo : hi;
                end[rows] = sum > 0 ? hi : lo;
                mult[rows] = (uint64_t)(sum > 0 ? sum : -sum);
            }
            ++rows;
        }
        i = j;
    }
    free(e);
    return rows;
}

/* Projection onto the plane orthogonal to the ray axis (detail/gwn_query_winding_antipodal_impl.cuh:
 * 54-63): x -> (y, z), y -> (z, x), z -> (x, y). */
static inline void ap_project(o_v3 v, int axis, float *px, float *py) {
    if (axis == 0) {
        *px = v.y;
        *py = v.z;
    } else if (axis == 1) {
        *px = v.z;
        *py = v.x;
    } else {
        *px = v.x;
        *py = v.y;
    }
}

static inline int ap_sign(float v) { return v > 0.0f ? 1 : (v < 0.0f ? -1 : 0); }

/* :76-111: projected determinant, its sign with the lexicographic symbolic perturbation, and the
 * singular flag of a collinear edge whose endpoints lie on opposite sides of the query. */
static inline void ap_classify(o_v3 s, o_v3 e, int axis, int *sign, int *singular, float *det) {
    float ax, ay, bx, by;
    ap_project(s, axis, &ax, &ay);
    ap_project(e, axis, &bx, &by);
    float const d = o_dop(ax, by, ay, bx);
    int sg = ap_sign(d);
    if (sg == 0) {
        sg = ap_sign(ay - by);
        if (sg == 0)
            sg = ap_sign(bx - ax);
    }
    *sign = sg;
    *det = d;
    *singular = d == 0.0f && fmaf(ay, by, ax * bx) <= 0.0f;
}

static inline float ap_axis_component(o_v3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

/* :123-177: crossing sign of one oriented triangle with the positive axis ray; 1 when singular. */
static int ap_triangle_crossing(o_v3 q, int axis, o_v3 a, o_v3 b, o_v3 c, float *crossing) {
    o_v3 const pa = v3_sub(a, q), pb = v3_sub(b, q), pc = v3_sub(c, q);
    o_v3 const n = v3_cross(v3_sub(pb, pa), v3_sub(pc, pa));
    float const na = ap_axis_component(n, axis);
    if (na == 0.0f)
        return 0;
    int s0, s1, s2, g0, g1, g2;
    float d;
    ap_classify(pa, pb, axis, &s0, &g0, &d);
    ap_classify(pb, pc, axis, &s1, &g1, &d);
    ap_classify(pc, pa, axis, &s2, &g2, &d);
    if (g0 || g1 || g2)
        return 1;
    if (s0 == 0 || s1 == 0 || s2 == 0)
        return 1;
    if (!((s0 >= 0 && s1 >= 0 && s2 >= 0) || (s0 <= 0 && s1 <= 0 && s2 <= 0)))
        return 0;
    float const t = v3_dot(n, pa) / na;
    if (t == 0.0f)
        return 1;
    if (!(t > 0.0f))
        return 0;
    *crossing += na > 0.0f ? 1.0f : -1.0f;
    return 0;
}

/* :380-489: signed crossings of the positive axis ray through the canonical BVH (children in slot
 * order, leaves evaluated in place, the last internal child entered directly). Returns 1 when
 * singular, 2 on stack overflow. */
static int ap_crossings(const o_node4 *nodes, uint64_t nn, const o_tri *tris, uint64_t nt, uint64_t root_ref, o_v3 q,
                        int axis, int cap, float *sum) {
    float const qc[3] = {q.x, q.y, q.z};
    int const u = axis == 0 ? 1 : (axis == 1 ? 2 : 0), w = axis == 0 ? 2 : (axis == 1 ? 0 : 1);
    *sum = 0.0f;
#define AP_LEAF(R)                                                                                  \
    for (uint32_t k_ = 0; k_ < ref_count(R); ++k_) {                                                \
        uint64_t const si_ = ref_offset(R) + k_;                                                    \
        if (si_ >= nt)                                                                              \
            continue;                                                                               \
        o_v3 a_, b_, c_;                                                                            \
        record_vertices(&tris[si_], &a_, &b_, &c_);                                                 \
        if (ap_triangle_crossing(q, axis, a_, b_, c_, sum))                                          \
            return 1;                                                                               \
    }
    if (ref_leaf(root_ref)) {
        AP_LEAF(root_ref)
        return 0;
    }
    uint32_t stack[256];
    int sp = 0;
    uint64_t node = ref_offset(root_ref);
    for (;;) {
        uint64_t next = (uint64_t)-1;
        if (node < nn) {
            const o_node4 *nd = &nodes[node];
            for (int s = 0; s < 4; ++s) {
                uint64_t const r = nd->c[s].reference;
                if (!ref_valid(r))
                    continue;
                const o_aabb *b = &nd->c[s].bounds;
                float const lo[3] = {b->min_x, b->min_y, b->min_z}, hi[3] = {b->max_x, b->max_y, b->max_z};
                if (!(qc[u] >= lo[u] && qc[u] <= hi[u] && qc[w] >= lo[w] && qc[w] <= hi[w] && hi[axis] >= qc[axis]))
                    continue;
                if (ref_leaf(r)) {
                    AP_LEAF(r)
                    continue;
                }
                if (!ref_internal(r))
                    continue;
                if (next != (uint64_t)-1) {
                    if (sp >= cap)
                        return 2;
                    stack[sp++] = (uint32_t)next;
                }
                next = ref_offset(r);
            }
        }
        if (next != (uint64_t)-1) {
            node = next;
            continue;
        }
        if (sp == 0)
            break;
        node = stack[--sp];
    }
#undef AP_LEAF
    return 0;
}

static const double ap_pi = 3.141592653589793238462643383279502884;

/* Terms whose atan2 arguments are both below this fraction of |s||e| are evaluated in FP64: the
 * edge passes close to the ray line seen from the query, the term (and its gradient, which grows
 * like the inverse of that distance) is dominated by float rounding there, and neighbouring terms
 * of that size cancel. The decision is made on the float values, identically on the GPU. */
static const float ap_guard = 1.0f / 16.0f;

static inline int ap_guarded(float num, float den, float ls, float le) {
    float const sl = ls * le;
    return fmaf(den, den, num * num) < (ap_guard * ap_guard) * (sl * sl);
}

/* The term's vectors in FP64 from the float end points and query. */
static inline void ap_vectors_d(o_v3 S, o_v3 E, o_v3 q, double s[3], double e[3]) {
    s[0] = (double)S.x - (double)q.x;
    s[1] = (double)S.y - (double)q.y;
    s[2] = (double)S.z - (double)q.z;
    e[0] = (double)E.x - (double)q.x;
    e[1] = (double)E.y - (double)q.y;
    e[2] = (double)E.z - (double)q.z;
}

/* -ray . (s x e), |s|, |e| and the atan2 denominator in FP64. */
static inline void ap_terms_d(int axis, const double s[3], const double e[3], double *num, double *den, double *ls,
                              double *le) {
    double const c[3] = {s[1] * e[2] - s[2] * e[1], s[2] * e[0] - s[0] * e[2], s[0] * e[1] - s[1] * e[0]};
    *ls = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    *le = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    *num = -c[axis];
    *den = *ls * *le - s[axis] * *le - e[axis] * *ls + (s[0] * e[0] + s[1] * e[1] + s[2] * e[2]);
}

/* :188-205: signed spherical area of (-ray, edge start, edge end), 2 atan2(numerator, denominator);
 * for guarded terms the atan2 arguments come from FP64 vectors (S, E and q). */
static double ap_area(int axis, o_v3 mr, o_v3 s, o_v3 e, float det, o_v3 S, o_v3 E, o_v3 q, int *guarded) {
    float const ls = sqrtf(v3_dot(s, s)), le = sqrtf(v3_dot(e, e));
    *guarded = 0;
    if (!(ls > 0.0f) || !(le > 0.0f))
        return NAN;
    float num = -det;
    if (det == 0.0f)
        num = v3_dot(mr, v3_cross(s, e));
    float const den = fmaf(v3_dot(e, mr), ls, fmaf(v3_dot(mr, s), le, ls * le) + v3_dot(s, e));
    if (ap_guarded(num, den, ls, le)) {
        /* the angle of accurately known arguments is well conditioned: atan2 in float suffices */
        double sd[3], ed[3], nd, dd, lsd, led;
        ap_vectors_d(S, E, q, sd, ed);
        ap_terms_d(axis, sd, ed, &nd, &dd, &lsd, &led);
        *guarded = 1;
        return (double)(2.0f * atan2f((float)nd, (float)dd));
    }
    return (double)(2.0f * atan2f(num, den));
}

/* Edge records (start, end, multiplicity) gathered from the geometry. */
static inline void ap_edge(const float *vx, const float *vy, const float *vz, uint32_t a, uint32_t b, o_v3 q, o_v3 *s,
                           o_v3 *e) {
    *s = v3(vx[a] - q.x, vy[a] - q.y, vz[a] - q.z);
    *e = v3(vx[b] - q.x, vy[b] - q.y, vz[b] - q.z);
}

/* :209-256: boundary term of one axis, summed in FP64 in row order. Returns 1 when singular. */
static int ap_boundary(const float *vx, const float *vy, const float *vz, const uint32_t *start, const uint32_t *end,
                       const uint64_t *mult, uint64_t ne, o_v3 q, int axis, double *out) {
    o_v3 mr = v3(0.0f, 0.0f, 0.0f);
    if (axis == 0)
        mr.x = -1.0f;
    else if (axis == 1)
        mr.y = -1.0f;
    else
        mr.z = -1.0f;
    double sum = 0.0;
    for (uint64_t i = 0; i < ne; ++i) {
        o_v3 s, e;
        ap_edge(vx, vy, vz, start[i], end[i], q, &s, &e);
        int sign, singular;
        float det;
        ap_classify(s, e, axis, &sign, &singular, &det);
        if (singular)
            return 1;
        o_v3 const S = v3(vx[start[i]], vy[start[i]], vz[start[i]]), E = v3(vx[end[i]], vy[end[i]], vz[end[i]]);
        int guarded;
        float area = (float)ap_area(axis, mr, s, e, det, S, E, q, &guarded);
        if (axis != 2 && sign > 0 && area < 0.0f)
            area += (float)(2.0 * ap_pi);
        sum += (double)((float)mult[i] * area);
    }
    *out = sum / (4.0 * ap_pi);
    return 0;
}

/* :533-568 (z, then x, then y): crossings plus boundary term of the first axis on which neither is
 * singular; NaN when all three are (or on stack overflow). */
void oracle_antipodal(const float *vx, const float *vy, const float *vz, const o_node4 *nodes, uint64_t nn,
                      const o_tri *tris, uint64_t nt, uint64_t root_ref, const uint32_t *start, const uint32_t *end,
                      const uint64_t *mult, uint64_t ne, const float *qx, const float *qy, const float *qz, uint64_t n,
                      int stack_capacity, float *out, int threads) {
    int const cap = stack_capacity > 256 ? 256 : stack_capacity;
    static const int order[3] = {2, 0, 1};
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        o_v3 const q = v3(qx[i], qy[i], qz[i]);
        float result = NAN;
        for (int k = 0; k < 3; ++k) {
            float cross;
            int const c = ap_crossings(nodes, nn, tris, nt, root_ref, q, order[k], cap, &cross);
            if (c == 2)
                break;
            if (c == 1)
                continue;
            double b;
            if (ap_boundary(vx, vy, vz, start, end, mult, ne, q, order[k], &b))
                continue;
            result = (float)((double)cross + b);
            break;
        }
        out[i] = result;
    }
}

static inline o_v3 v3_scale(o_v3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }

/* The same gradient in FP64 (guarded terms). */
static void ap_area_gradient_d(int axis, o_v3 S, o_v3 E, o_v3 q, double g[3]) {
    double s[3], e[3], num, den, ls, le;
    ap_vectors_d(S, E, q, s, e);
    ap_terms_d(axis, s, e, &num, &den, &ls, &le);
    double mr[3] = {0.0, 0.0, 0.0};
    mr[axis] = -1.0;
    double const d2 = num * num + den * den;
    if (ls == 0.0 || le == 0.0 || d2 == 0.0) {
        g[0] = g[1] = g[2] = NAN;
        return;
    }
    double su[3], eu[3];
    for (int k = 0; k < 3; ++k) {
        su[k] = s[k] / ls;
        eu[k] = e[k] / le;
    }
    double const cn = 2.0 * den / d2, cd = -2.0 * num / d2;
    double const me = mr[0] * eu[0] + mr[1] * eu[1] + mr[2] * eu[2];
    double const ms = mr[0] * su[0] + mr[1] * su[1] + mr[2] * su[2];
    /* e x mr + mr x s */
    double const gn[3] = {-((e[1] * mr[2] - e[2] * mr[1]) + (mr[1] * s[2] - mr[2] * s[1])),
                          -((e[2] * mr[0] - e[0] * mr[2]) + (mr[2] * s[0] - mr[0] * s[2])),
                          -((e[0] * mr[1] - e[1] * mr[0]) + (mr[0] * s[1] - mr[1] * s[0]))};
    for (int k = 0; k < 3; ++k) {
        double const t1 = le * (mr[k] + eu[k] + (1.0 + me) * su[k]);
        double const t2 = ls * (mr[k] + su[k] + (1.0 + ms) * eu[k]);
        g[k] = cn * gn[k] - cd * (t1 + t2);
    }
}

/* :261-304: gradient of one signed spherical-area term with respect to the query; FP64 for guarded
 * terms (returned in gd with *guarded set). */
static o_v3 ap_area_gradient(int axis, o_v3 mr, o_v3 s, o_v3 e, float det, o_v3 S, o_v3 E, o_v3 q, int *guarded,
                             double gd_out[3]) {
    o_v3 const nan3 = v3(NAN, NAN, NAN);
    *guarded = 0;
    float const ls = sqrtf(v3_dot(s, s)), le = sqrtf(v3_dot(e, e));
    if (ls == 0.0f || le == 0.0f)
        return nan3;
    o_v3 const su = v3_scale(s, 1.0f / ls), eu = v3_scale(e, 1.0f / le);
    float num = -det;
    if (det == 0.0f)
        num = v3_dot(mr, v3_cross(s, e));
    float const den = fmaf(v3_dot(mr, e), ls, fmaf(v3_dot(mr, s), le, ls * le) + v3_dot(s, e));
    if (ap_guarded(num, den, ls, le)) {
        *guarded = 1;
        ap_area_gradient_d(axis, S, E, q, gd_out);
        return nan3;
    }
    float const d2 = fmaf(den, den, num * num);
    if (d2 == 0.0f)
        return nan3;
    float const cn = 2.0f * den / d2, cd = -2.0f * num / d2;
    o_v3 const gn = v3_scale(v3_add(v3_cross(e, mr), v3_cross(mr, s)), -1.0f);
    o_v3 const t1 = v3_scale(v3_fma(su, 1.0f + v3_dot(mr, eu), v3_add(mr, eu)), le);
    o_v3 const t2 = v3_scale(v3_fma(eu, 1.0f + v3_dot(mr, su), v3_add(mr, su)), ls);
    o_v3 const gd = v3_scale(v3_add(t1, t2), -1.0f);
    return v3_fma(gd, cd, v3_scale(gn, cn));
}

/* :307-372: gradient of the boundary term (FP64 sums), axis retries z, x, y; NaN when all three
 * are singular. */
void oracle_antipodal_gradient(const float *vx, const float *vy, const float *vz, const uint32_t *start,
                               const uint32_t *end, const uint64_t *mult, uint64_t ne, const float *qx,
                               const float *qy, const float *qz, uint64_t n, float *gx, float *gy, float *gz,
                               int threads) {
    static const int order[3] = {2, 0, 1};
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        o_v3 const q = v3(qx[i], qy[i], qz[i]);
        float r[3] = {NAN, NAN, NAN};
        for (int k = 0; k < 3; ++k) {
            int const axis = order[k];
            o_v3 mr = v3(0.0f, 0.0f, 0.0f);
            if (axis == 0)
                mr.x = -1.0f;
            else if (axis == 1)
                mr.y = -1.0f;
            else
                mr.z = -1.0f;
            double sx = 0.0, sy = 0.0, sz = 0.0;
            int singular = 0;
            for (uint64_t j = 0; j < ne && !singular; ++j) {
                o_v3 s, e;
                ap_edge(vx, vy, vz, start[j], end[j], q, &s, &e);
                int sign;
                float det;
                ap_classify(s, e, axis, &sign, &singular, &det);
                if (singular)
                    break;
                o_v3 const S = v3(vx[start[j]], vy[start[j]], vz[start[j]]);
                o_v3 const E = v3(vx[end[j]], vy[end[j]], vz[end[j]]);
                int guarded;
                double gd[3];
                o_v3 const g = ap_area_gradient(axis, mr, s, e, det, S, E, q, &guarded, gd);
                if (guarded) {
                    double const md = (double)mult[j];
                    sx += md * gd[0];
                    sy += md * gd[1];
                    sz += md * gd[2];
                } else {
                    float const m = (float)mult[j];
                    sx += (double)(m * g.x);
                    sy += (double)(m * g.y);
                    sz += (double)(m * g.z);
                }
            }
            if (singular)
                continue;
            double const k4 = 4.0 * ap_pi;
            r[0] = (float)(sx / k4);
            r[1] = (float)(sy / k4);
            r[2] = (float)(sz / k4);
            break;
        }
        gx[i] = r[0];
        gy[i] = r[1];
        gz[i] = r[2];
    }
}
