// Near-field (exact solid angle) and far-field (Taylor) terms of the winding number, shared by the
// query and adjoint translation units.
//
// Solid angle of a triangle seen from q: the Van Oosterom-Strackee formula in unnormalised form,
// tan(Omega/2) = a.(e1 x e2) / (|a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a|) with a = v0 - q,
// b = a + e1, c = a + e2; it equals smallgwn's unit-vector form
// (detail/gwn_query_geometry_impl.cuh:16-45) and keeps its conventions: zero when the query sits on
// a vertex or the numerator vanishes.
//
// Far field of one child slot: smallgwn's expansion (detail/gwn_query_winding_impl.cuh:193-327)
// about the slot's area-weighted centre P with r = q - P: order 0 -(r.N)/|r|^3, order 1
// (tr M - 3 r^T M r / |r|^2) / |r|^3 with M_ij = sum n_i (c - P)_j, order 2 the third-moment terms.
#pragma once

#include "gwnb_internal.cuh"

namespace gwnb {
namespace field {

constexpr float k_pi_f = 3.14159265358979323846f;

// |q - P|^2 for the acceptance test, with one fixed rounding pattern (rx * rx rounded, then two
// fused multiply-adds) written out so that no compiler contraction choice can change it. Every
// traversal (value, gradient, statistics, adjoint, batched) and the oracle's C restatement use
// this pattern, so their accept / descend decisions are identical for identical inputs.
__device__ __forceinline__ float accept_dist2(float rx, float ry, float rz) {
    return __fmaf_rn(rz, rz, __fmaf_rn(ry, ry, __fmul_rn(rx, rx)));
}

// smallgwn's acceptance rule (detail/gwn_query_winding_impl.cuh:186-189): descend iff
// !(|q - P|^2 > 0) or |q - P|^2 <= r^2 beta^2 (the product rounded on its own); a NaN bound
// therefore accepts, as there.
__device__ __forceinline__ bool far_accepted(float q2, float r2, float beta2) {
    return q2 > 0.0f && !(q2 <= __fmul_rn(r2, beta2));
}

// a = v0 - q, e1, e2 edges, n = e1 x e2.
__device__ __forceinline__ float solid_angle_plain(float ax, float ay, float az, float e1x, float e1y,
                                                   float e1z, float e2x, float e2y, float e2z,
                                                   float nx, float ny, float nz) {
    float const bx = ax + e1x, by = ay + e1y, bz = az + e1z;
    float const cx = ax + e2x, cy = ay + e2y, cz = az + e2z;
    float const a2 = ax * ax + ay * ay + az * az;
    float const b2 = bx * bx + by * by + bz * bz;
    float const c2 = cx * cx + cy * cy + cz * cz;
    float const la = sqrtf(a2), lb = sqrtf(b2), lc = sqrtf(c2);
    if (la == 0.0f || lb == 0.0f || lc == 0.0f)
        return 0.0f;
    float const num = ax * nx + ay * ny + az * nz;
    if (num == 0.0f)
        return 0.0f;
    float const ab = ax * bx + ay * by + az * bz;
    float const ac = ax * cx + ay * cy + az * cz;
    float const bc = bx * cx + by * cy + bz * cz;
    float const den = la * lb * lc + ab * lc + ac * lb + bc * la;
    return 2.0f * atan2f(num, den);
}

// Error-free transformations (Dekker / Ogita-Rump-Oishi "Accurate sum and dot product", 2005).
__device__ __forceinline__ void two_prod(float a, float b, float &p, float &e) {
    p = a * b;
    e = fmaf(a, b, -p);
}
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = a + b;
    float const z = s - a;
    e = (a - (s - z)) + (b - z);
}
// Compensated dot product of length 3 (Dot2).
__device__ __forceinline__ float dot3_comp(float a0, float a1, float a2, float b0, float b1, float b2) {
    float p, s, h, r, q;
    two_prod(a0, b0, p, s);
    two_prod(a1, b1, h, r);
    two_sum(p, h, p, q);
    s += q + r;
    two_prod(a2, b2, h, r);
    two_sum(p, h, p, q);
    s += q + r;
    return p + s;
}

// FP64 evaluation of one (query, triangle) pair over the same float record (b = a + e1 and
// c = a + e2 are exact in double), for pairs whose numerator and denominator both cancel.
__device__ __forceinline__ float solid_angle_f64_fallback(float ax, float ay, float az, float e1x,
                                                          float e1y, float e1z, float e2x, float e2y,
                                                          float e2z, unsigned long long *fp64_count) {
    if (fp64_count != nullptr)
        atomicAdd(fp64_count, 1ull);
    double const dax = ax, day = ay, daz = az;
    double const dbx = dax + e1x, dby = day + e1y, dbz = daz + e1z;
    double const dcx = dax + e2x, dcy = day + e2y, dcz = daz + e2z;
    double const dla = sqrt(dax * dax + day * day + daz * daz);
    double const dlb = sqrt(dbx * dbx + dby * dby + dbz * dbz);
    double const dlc = sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
    double const dnx = static_cast<double>(e1y) * e2z - static_cast<double>(e1z) * e2y;
    double const dny = static_cast<double>(e1z) * e2x - static_cast<double>(e1x) * e2z;
    double const dnz = static_cast<double>(e1x) * e2y - static_cast<double>(e1y) * e2x;
    double const dnum = dax * dnx + day * dny + daz * dnz;
    if (dnum == 0.0)
        return 0.0f;
    double const dden = dla * dlb * dlc + (dax * dbx + day * dby + daz * dbz) * dlc +
                        (dax * dcx + day * dcy + daz * dcz) * dlb +
                        (dbx * dcx + dby * dcy + dbz * dcz) * dla;
    return static_cast<float>(2.0 * atan2(dnum, dden));
}

// Exact-batch form: the plain FP32 evaluation, except that pairs with both |num| and |den| below
// |a||b||c| / 16 -- a query within a small angle of an edge's line or at a vertex, where FP32
// cancellation leaves errors up to ~1e-3 -- are evaluated in FP64. On near-surface query sets
// about 0.1 pairs per query take that branch.
constexpr float k_exact_guard = 1.0f / 16.0f;

__device__ __forceinline__ float solid_angle_guarded(float ax, float ay, float az, float e1x, float e1y,
                                                     float e1z, float e2x, float e2y, float e2z,
                                                     float nx, float ny, float nz) {
    float const bx = ax + e1x, by = ay + e1y, bz = az + e1z;
    float const cx = ax + e2x, cy = ay + e2y, cz = az + e2z;
    float const a2 = ax * ax + ay * ay + az * az;
    float const b2 = bx * bx + by * by + bz * bz;
    float const c2 = cx * cx + cy * cy + cz * cz;
    if (a2 == 0.0f || b2 == 0.0f || c2 == 0.0f)
        return 0.0f;
    // lengths as x * rsqrt(x) (within 2 ulp of the rounded square root): the brute-force batch
    // evaluates every pair, and the pairs it cannot take in float go to the FP64 branch below
    float const la = a2 * rsqrtf(a2), lb = b2 * rsqrtf(b2), lc = c2 * rsqrtf(c2);
    float const num = ax * nx + ay * ny + az * nz;
    float const labc = la * lb * lc;
    float const den = labc + (ax * bx + ay * by + az * bz) * lc + (ax * cx + ay * cy + az * cz) * lb +
                      (bx * cx + by * cy + bz * cz) * la;
    float const lim = k_exact_guard * labc;
    if (fabsf(num) < lim && fabsf(den) < lim)
        return solid_angle_f64_fallback(ax, ay, az, e1x, e1y, e1z, e2x, e2y, e2z, nullptr);
    if (num == 0.0f)
        return 0.0f;
    return 2.0f * atan2f(num, den);
}

// Compensated near field (Taylor traversal): the two atan2 arguments -- the triple product
// a.(e1 x e2) and the denominator's sum |a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a| -- as compensated
// (Dot2) sums; pairs whose numerator and denominator are both below threshold * |a||b||c| take the
// FP64 evaluation. The rounding of b = a + e1 and c = a + e2 themselves bounds what compensation can
// recover (the FP64 branch removes it), so the three inner dot products stay plain FP32.
__device__ __forceinline__ float solid_angle_comp(float ax, float ay, float az, float e1x, float e1y,
                                                  float e1z, float e2x, float e2y, float e2z, float nx,
                                                  float ny, float nz, float threshold,
                                                  unsigned long long *fp64_count) {
    // Lengths are sums of squares (no cancellation): plain FP32. n = e1 x e2 is the record's.
    float const bx = ax + e1x, by = ay + e1y, bz = az + e1z;
    float const cx = ax + e2x, cy = ay + e2y, cz = az + e2z;
    float const la = sqrtf(ax * ax + ay * ay + az * az);
    float const lb = sqrtf(bx * bx + by * by + bz * bz);
    float const lc = sqrtf(cx * cx + cy * cy + cz * cz);
    if (la == 0.0f || lb == 0.0f || lc == 0.0f)
        return 0.0f;
    float const num = dot3_comp(ax, ay, az, nx, ny, nz);
    float const ab = ax * bx + ay * by + az * bz;
    float const ac = ax * cx + ay * cy + az * cz;
    float const bc = bx * cx + by * cy + bz * cz;
    float const labc = la * lb * lc;
    float const den = labc + dot3_comp(ab, ac, bc, lc, lb, la);
    float const scale = labc;
    if (fabsf(den) < threshold * scale && fabsf(num) < threshold * scale)
        return solid_angle_f64_fallback(ax, ay, az, e1x, e1y, e1z, e2x, e2y, e2z, fp64_count);
    if (num == 0.0f)
        return 0.0f;
    return 2.0f * atan2f(num, den);
}

// Gradient of the solid angle w.r.t. the query (Biot-Savart form), as smallgwn's
// gwn_gradient_solid_angle_triangle_impl (detail/gwn_query_winding_impl.cuh:21-60).
__device__ __forceinline__ float3 solid_angle_grad(float ax, float ay, float az, float e1x, float e1y,
                                                   float e1z, float e2x, float e2y, float e2z) {
    float3 const g[3] = {make_float3(ax, ay, az), make_float3(ax + e1x, ay + e1y, az + e1z),
                         make_float3(ax + e2x, ay + e2y, az + e2z)};
    float l[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        l[i] = sqrtf(g[i].x * g[i].x + g[i].y * g[i].y + g[i].z * g[i].z);
    if (l[0] == 0.0f || l[1] == 0.0f || l[2] == 0.0f)
        return make_float3(0.0f, 0.0f, 0.0f);
    float3 h[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        h[i] = make_float3(g[i].x / l[i], g[i].y / l[i], g[i].z / l[i]);
    float3 r = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        int const i = e, j = (e + 1) % 3;
        float3 const cr = make_float3(g[i].y * g[j].z - g[i].z * g[j].y, g[i].z * g[j].x - g[i].x * g[j].z,
                                      g[i].x * g[j].y - g[i].y * g[j].x);
        float const cs = cr.x * cr.x + cr.y * cr.y + cr.z * cr.z;
        if (cs == 0.0f)
            continue;
        float const sc = ((g[i].x - g[j].x) * (h[i].x - h[j].x) + (g[i].y - g[j].y) * (h[i].y - h[j].y) +
                          (g[i].z - g[j].z) * (h[i].z - h[j].z)) /
                         cs;
        r.x += sc * cr.x;
        r.y += sc * cr.y;
        r.z += sc * cr.z;
    }
    return r;
}

// Derivatives of the solid angle with respect to the three vertex offsets a = v0 - q, b = v1 - q,
// c = v2 - q. With Omega = 2 atan2(N, D), N = a.(b x c) and D = |a||b||c| + (a.b)|c| + (a.c)|b| +
// (b.c)|a|: dOmega = 2 (D dN - N dD) / (N^2 + D^2), where
//   dN/da = b x c,  dN/db = c x a,  dN/dc = a x b,
//   dD/da = a^ (|b||c| + b.c) + b|c| + c|b|  (and cyclically for b, c).
// The derivative with respect to the query is -(d/da + d/db + d/dc). Zero when the query sits on a
// vertex or N = D = 0.
struct vertex_grad {
    float3 a, b, c;
};

__device__ __forceinline__ vertex_grad solid_angle_vertex_grad(float ax, float ay, float az, float e1x,
                                                               float e1y, float e1z, float e2x, float e2y,
                                                               float e2z) {
    vertex_grad r{};
    float const bx = ax + e1x, by = ay + e1y, bz = az + e1z;
    float const cx = ax + e2x, cy = ay + e2y, cz = az + e2z;
    float const la = sqrtf(ax * ax + ay * ay + az * az);
    float const lb = sqrtf(bx * bx + by * by + bz * bz);
    float const lc = sqrtf(cx * cx + cy * cy + cz * cz);
    if (la == 0.0f || lb == 0.0f || lc == 0.0f)
        return r;
    // cross products b x c, c x a, a x b
    float const bcx = by * cz - bz * cy, bcy = bz * cx - bx * cz, bcz = bx * cy - by * cx;
    float const cax = cy * az - cz * ay, cay = cz * ax - cx * az, caz = cx * ay - cy * ax;
    float const abx = ay * bz - az * by, aby = az * bx - ax * bz, abz = ax * by - ay * bx;
    float const N = ax * bcx + ay * bcy + az * bcz;
    float const dab = ax * bx + ay * by + az * bz;
    float const dac = ax * cx + ay * cy + az * cz;
    float const dbc = bx * cx + by * cy + bz * cz;
    float const D = la * lb * lc + dab * lc + dac * lb + dbc * la;
    float const s = N * N + D * D;
    if (!(s > 0.0f))
        return r;
    float const kD = 2.0f * D / s;
    float const kN = 2.0f * N / s;
    float const fa = (lb * lc + dbc) / la, fb = (la * lc + dac) / lb, fc = (la * lb + dab) / lc;
    r.a.x = kD * bcx - kN * (fa * ax + bx * lc + cx * lb);
    r.a.y = kD * bcy - kN * (fa * ay + by * lc + cy * lb);
    r.a.z = kD * bcz - kN * (fa * az + bz * lc + cz * lb);
    r.b.x = kD * cax - kN * (fb * bx + ax * lc + cx * la);
    r.b.y = kD * cay - kN * (fb * by + ay * lc + cy * la);
    r.b.z = kD * caz - kN * (fb * bz + az * lc + cz * la);
    r.c.x = kD * abx - kN * (fc * cx + ax * lb + bx * la);
    r.c.y = kD * aby - kN * (fc * cy + ay * lb + by * la);
    r.c.z = kD * abz - kN * (fc * cz + az * lb + bz * la);
    return r;
}

// Far-field Taylor terms of one accepted child: smallgwn's expansion
// (gwn_query_winding_impl.cuh:193-327) on the folded sidecar coefficients the moment refit writes.
// r = q - P, q2 = |r|^2, n = r / |r|; b = (N, ref); cd.. = order-1 quadratic form M' (xx yy zz xy yz
// zx) then order-2 cubic form K (xxx yyy zzz xxy xxz yyx yyz zzx zzy xyz):
//   w = -(n.N) / |r|^2 + n^T M' n / |r|^3 + K(n,n,n) / |r|^4.
// With Grad, g is the derivative with respect to the query: the terms are P(r) / |r|^(2p+1) for
// homogeneous P of degree p = 1, 2, 3, whose gradient is (grad P(n) - (2p+1) P(n) n) / |r|^(p+2).
template <int Order, bool Grad>
__device__ __forceinline__ float far_field(float rx, float ry, float rz, float q2, float4 const &b,
                                           float4 const *__restrict__ cd, float &g0, float &g1, float &g2) {
    float const m1 = rsqrtf(q2);
    float const m2 = m1 * m1;
    float const m3 = m2 * m1;
    float const nx = rx * m1, ny = ry * m1, nz = rz * m1;
    float const rdn = nx * b.x + ny * b.y + nz * b.z;
    float w = -m2 * rdn;
    if constexpr (Grad) {
        g0 = m3 * (3.0f * nx * rdn - b.x);
        g1 = m3 * (3.0f * ny * rdn - b.y);
        g2 = m3 * (3.0f * nz * rdn - b.z);
    }
    if constexpr (Order >= 1 && !Grad) {
        // value only: the forms factored by components (Q1 in 7 and Q2 in 13 operations on the
        // shared squares), grouped explicitly since the compiler keeps the written FP order
        float4 const c = __ldg(cd);
        float4 const d = __ldg(cd + 1);
        float const xx = nx * nx, yy = ny * ny, zz = nz * nz, yz = ny * nz;
        float const Q1 = c.x * xx + c.y * yy + c.z * zz + d.x * yz + nx * (c.w * ny + d.y * nz);
        float t = Q1;
        if constexpr (Order >= 2) {
            float4 const e = __ldg(cd + 2);
            float4 const f = __ldg(cd + 3);
            float const Q2 = nx * (d.z * xx + e.w * yy + f.y * zz + f.w * yz) + ny * (d.w * yy + e.y * xx + f.z * zz) +
                             nz * (e.x * zz + e.z * xx + f.x * yy);
            t += m1 * Q2;
        }
        w += m3 * t;
        return w;
    }
    if constexpr (Order >= 1) {
        float4 const c = __ldg(cd);
        float4 const d = __ldg(cd + 1);
        float const xx = nx * nx, yy = ny * ny, zz = nz * nz, xy = nx * ny, yz = ny * nz, zx = nz * nx;
        float const Q1 = c.x * xx + c.y * yy + c.z * zz + c.w * xy + d.x * yz + d.y * zx;
        w += m3 * Q1;
        if constexpr (Grad) {
            float const m4 = m2 * m2;
            float const k = 5.0f * Q1;
            g0 += m4 * (2.0f * c.x * nx + c.w * ny + d.y * nz - k * nx);
            g1 += m4 * (c.w * nx + 2.0f * c.y * ny + d.x * nz - k * ny);
            g2 += m4 * (d.y * nx + d.x * ny + 2.0f * c.z * nz - k * nz);
        }
        if constexpr (Order >= 2) {
            float4 const e = __ldg(cd + 2);
            float4 const f = __ldg(cd + 3);
            // K over xxx yyy zzz xxy | xxz yyx yyz zzx | zzy xyz
            float const Q2 = d.z * xx * nx + d.w * yy * ny + e.x * zz * nz + e.y * xx * ny + e.z * xx * nz +
                             e.w * yy * nx + f.x * yy * nz + f.y * zz * nx + f.z * zz * ny + f.w * xy * nz;
            float const m4 = m2 * m2;
            w += m4 * Q2;
            if constexpr (Grad) {
                float const m5 = m4 * m1;
                float const k = 7.0f * Q2;
                float const Gx = 3.0f * d.z * xx + 2.0f * e.y * xy + 2.0f * e.z * zx + e.w * yy + f.y * zz + f.w * yz;
                float const Gy = 3.0f * d.w * yy + e.y * xx + 2.0f * e.w * xy + 2.0f * f.x * yz + f.z * zz + f.w * zx;
                float const Gz = 3.0f * e.x * zz + e.z * xx + f.x * yy + 2.0f * f.y * zx + 2.0f * f.z * yz + f.w * xy;
                g0 += m5 * (Gx - k * nx);
                g1 += m5 * (Gy - k * ny);
                g2 += m5 * (Gz - k * nz);
            }
        }
    }
    return w;
}

} // namespace field
} // namespace gwnb
