"""FP64 explanations of Taylor disagreements between two implementations over the same tree.

Two Taylor batches over structurally identical BVH4s (same slot order; node numbering may differ)
and their own moment nodes can disagree beyond rounding for two reasons only:

- a **decision**: some child's acceptance test (detail/gwn_query_winding_impl.cuh:186-189, accept
  iff |q - P|^2 > r^2 beta^2) decides differently, because the two moment sets' P and r^2 differ
  in their last bits (their climbs sum in different orders) or because the float |q - P|^2 sits
  within rounding of the threshold; the query then moves by the local truncation error;
- **conditioning**: a triangle evaluated exactly in the near field is seen from a point close to
  the line of one of its edges, where both atan2 arguments of the solid angle (the triple product
  and |a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a|) cancel to below 1/16 of |a||b||c| and an FP32
  evaluation loses digits.

- **moments**: the two moment sets themselves differ. Order-2 coefficients are raw moments about
  the origin recentred at P (R - 2 P F + P^2 N, detail/gwn_bvh_refit_common.cuh:123-387), which
  cancels for a small node far from the origin; two FP32 climbs that sum in different orders then
  carry different coefficients. Evaluating the accepted far fields of the query in FP64 from each
  side's float moments reproduces the disagreement.

`explain` walks tree A depth first for one query, evaluating every child test in FP64 under both
moment sets, and reports which of these (if any) it finds. A disagreement that none explains is a
real parity failure.
"""
from __future__ import annotations

import numpy as np

VALID = 1 << 47
OFFSET_MASK = (1 << 47) - 1
CANCEL = 1.0 / 16.0


def _solid_angle_cancels(rec: np.ndarray, q: np.ndarray) -> bool:
    """Both atan2 arguments below 1/16 of the scale of the terms they are summed from: the
    triple product a.(e1 x e2) is bounded by |a||e1 x e2|, the denominator's terms by |a||b||c|."""
    v0 = rec[0:3].astype(np.float64)
    e1, e2 = rec[3:6].astype(np.float64), rec[6:9].astype(np.float64)
    a = v0 - q
    b, c = a + e1, a + e2
    la, lb, lc = np.linalg.norm(a), np.linalg.norm(b), np.linalg.norm(c)
    labc = la * lb * lc
    if labc == 0.0:
        return True
    n = np.cross(e1, e2)
    num = float(np.dot(a, n))
    den = labc + float(np.dot(a, b)) * lc + float(np.dot(a, c)) * lb + float(np.dot(b, c)) * la
    scale = max(labc, la * float(np.linalg.norm(n)))
    return abs(num) < CANCEL * scale and abs(den) < CANCEL * scale


def far_field64(mom: np.ndarray, k: int, s: int, q: np.ndarray) -> float:
    """smallgwn's far-field term of slot s of node k (detail/gwn_query_winding_impl.cuh:193-327) in FP64
    from the float moment fields (field-SoA layout: r^2, P, N, then 6 order-1 and 10 order-2 fields)."""
    f = mom[k, :, s].astype(np.float64)
    r = q - f[1:4]
    m1 = 1.0 / np.sqrt(float(r @ r))
    m2, m3 = m1 * m1, m1 * m1 * m1
    n = r * m1
    w = -m2 * float(n @ f[4:7])
    if f.size >= 13:
        xx, yy, zz, xy, yz, zx = f[7:13]
        S = n[0] ** 2 * xx + n[1] ** 2 * yy + n[2] ** 2 * zz + n[0] * n[1] * xy + n[0] * n[2] * zx + n[1] * n[2] * yz
        w += m3 * (xx + yy + zz - 3.0 * S)
    if f.size >= 23:
        xxx, yyy, zzz, spn, axy, axz, ayz, ayx, azx, azy = f[13:23]
        t0 = np.array([ayx + azx, azy + axy, axz + ayz])
        t1 = np.array([n[1] * axy + n[2] * axz, n[2] * ayz + n[0] * ayx, n[0] * azx + n[1] * azy])
        lin = n[0] * (3 * xxx + t0[0]) + n[1] * (3 * yyy + t0[1]) + n[2] * (3 * zzz + t0[2])
        cub = (n[0] ** 3 * xxx + n[1] ** 3 * yyy + n[2] ** 3 * zzz + n[0] * n[1] * n[2] * spn + n[0] ** 2 * t1[0] +
               n[1] ** 2 * t1[1] + n[2] ** 2 * t1[2])
        w += m2 * m2 * (1.5 * lin - 7.5 * cub)
    return float(w)


def explain(q, nodes_a: np.ndarray, root_ref: int, mom_a: np.ndarray, mom_b: np.ndarray, pairing: np.ndarray,
            tris_a: np.ndarray, beta: float, rel: float = 1e-6, observed: float = 0.0) -> str | None:
    """'decision', 'conditioning', 'moments' or None for query q = (x, y, z) (float32 values).

    nodes_a / tris_a: tree A's nodes and leaf-ordered triangle records; mom_a / mom_b: smallgwn-layout
    moment nodes (field 0 = r^2, fields 1-3 = P) of tree A and of tree B, with tree B's node
    pairing[i] corresponding to tree A's node i (None: the same numbering). `rel`: relative margin
    below which the float test may decide either way: |q - P|^2 carries three subtractions and
    three multiply(-add)s of relative rounding 2^-24 each, r^2 beta^2 one (together < 5e-7).
    `observed`: |a - b| of the two winding numbers; 'moments' when the FP64 far fields of the
    accepted slots, evaluated from each side's moments, differ by at least half of it."""
    qd = np.asarray(q, np.float64)
    beta2 = float(np.float32(np.float32(beta) * np.float32(beta)))
    nd = nodes_a.reshape(-1, 4)
    conditioning = False
    if (root_ref >> 48) != 0:
        first, cnt = root_ref & OFFSET_MASK, root_ref >> 48
        return "conditioning" if any(_solid_angle_cancels(tris_a[first + k], qd) for k in range(cnt)) else None
    stack = [root_ref & OFFSET_MASK]
    far_a = far_b = 0.0
    while stack:
        i = stack.pop()
        j = i if pairing is None else int(pairing[i])
        internal = []
        for s in range(4):
            r = int(nd[i, s]["reference"])
            if not r & VALID:
                continue
            decisions = []
            for mom, k in ((mom_a, i), (mom_b, j)):
                P = mom[k, 1:4, s].astype(np.float64)
                thr = float(mom[k, 0, s]) * beta2
                q2 = float(np.sum((qd - P) ** 2))
                if abs(q2 - thr) <= rel * max(thr, 1e-300):
                    return "decision"
                decisions.append(q2 > 0.0 and q2 > thr)
            if decisions[0] != decisions[1]:
                return "decision"
            if decisions[0]:
                if observed > 0.0 and mom_b is not mom_a:
                    far_a += far_field64(mom_a, i, s, qd)
                    far_b += far_field64(mom_b, j, s, qd)
                continue
            if (r >> 48) == 0:
                internal.append(r & OFFSET_MASK)
            else:
                first, cnt = r & OFFSET_MASK, r >> 48
                if any(_solid_angle_cancels(tris_a[first + k], qd) for k in range(cnt)):
                    conditioning = True
        # depth first in the kernels' order: the last internal child is entered next
        stack.extend(internal)
    if conditioning:
        return "conditioning"
    if observed > 0.0 and abs(far_a - far_b) / (4.0 * np.pi) >= 0.5 * observed:
        return "moments"
    return None


def disagreement_report(a: np.ndarray, b: np.ndarray, atol: float, rtol: float) -> dict:
    """Max and p99 of |a - b| over all queries and the indices outside atol + rtol * max(|a|, |b|)."""
    a64, b64 = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.abs(a64 - b64)
    bad = np.nonzero(d > atol + rtol * np.maximum(np.abs(a64), np.abs(b64)))[0]
    return {"max": float(d.max()) if d.size else 0.0, "p99": float(np.quantile(d, 0.99)) if d.size else 0.0,
            "outside": bad}
