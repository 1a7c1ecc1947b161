"""Record golden vectors from smallgwn's own CUDA implementation (oracle/_ref/libgwnref.so).

    python tests/golden/make_golden.py [out_dir]     # on a machine with a GPU

For each small fixture mesh this stores, from smallgwn's kernels on identical inputs: sorted
Morton codes (32- and 64-bit) and the sorted primitive permutation, the Karras LBVH binary
topology, the BVH4 built by gwn_build_bvh (LBVH and H-PLOC, r = 8) with its stack bounds and
triangle records, the H-PLOC binary topology as leaf sets, order 0/1/2 moments of the LBVH tree,
exact winding numbers, Taylor winding numbers (beta = 2 and beta = 1e6) and FP64 exact winding
numbers. tests/test_oracle.py checks the CPU restatement against these files, so the oracle is
pinned to the reference implementation without a GPU.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from smallgwn_b200 import meshes  # noqa: E402

OUT = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent


def fixture_meshes() -> dict[str, dict]:
    out = {}
    # asymmetric octahedron of smallgwn's query tests (tests/unit_gwn_query_winding.cu:23-30)
    out["asym_octahedron"] = {
        "x": np.array([1.7, -0.8, 0.15, -0.1, 0.2, -0.2], np.float32),
        "y": np.array([0.1, -0.2, 1.2, -0.7, 0.1, -0.1], np.float32),
        "z": np.array([0.0, 0.1, -0.1, 0.15, 1.5, -0.9], np.float32),
        "i0": np.array([0, 2, 1, 3, 2, 1, 3, 0], np.uint32),
        "i1": np.array([2, 1, 3, 0, 0, 2, 1, 3], np.uint32),
        "i2": np.array([4, 4, 4, 4, 5, 5, 5, 5], np.uint32),
    }
    # closed cube (tests/test_meshes.hpp:32-41)
    out["cube"] = {
        "x": np.array([-1, 1, 1, -1, -1, 1, 1, -1], np.float32),
        "y": np.array([-1, -1, 1, 1, -1, -1, 1, 1], np.float32),
        "z": np.array([-1, -1, -1, -1, 1, 1, 1, 1], np.float32),
        "i0": np.array([0, 0, 4, 4, 0, 0, 1, 1, 0, 0, 3, 3], np.uint32),
        "i1": np.array([2, 3, 5, 6, 4, 7, 2, 6, 1, 5, 7, 6], np.uint32),
        "i2": np.array([1, 2, 6, 7, 7, 3, 6, 5, 5, 4, 6, 2], np.uint32),
    }
    V, F = meshes.icosphere(2)
    out["icosphere2"] = meshes.to_soa(V, F)
    out["displaced_32x16"] = meshes.to_soa(*meshes.uv_sphere(32, 16, seed=7))
    out["soup_24"] = meshes.soup_mesh(24, seed=11)
    # equal bounds (tests/integration_gwn_builder.cu:301-343), 129 copies of one triangle
    out["equal_129"] = {
        "x": np.array([0, 1, 0], np.float32), "y": np.array([0, 0, 1], np.float32), "z": np.zeros(3, np.float32),
        "i0": np.zeros(129, np.uint32), "i1": np.ones(129, np.uint32), "i2": np.full(129, 2, np.uint32),
    }
    return out


def queries(mesh: dict, n: int = 64, seed: int = 5):
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=-1).astype(np.float64)
    lo, hi = P.min(0), P.max(0)
    c, h = (lo + hi) / 2, np.maximum((hi - lo) / 2, 1e-2) * 1.6
    rng = np.random.default_rng(seed)
    q = (c + rng.uniform(-1, 1, size=(n, 3)) * h).astype(np.float32)
    return tuple(np.ascontiguousarray(q[:, k]) for k in range(3))


def record(name: str, mesh: dict) -> None:
    R = oracle.Reference(mesh)
    qx, qy, qz = queries(mesh)
    rec: dict[str, np.ndarray] = {k: v for k, v in mesh.items()}
    rec.update(qx=qx, qy=qy, qz=qz)
    for bits in (32, 64):
        codes, ids, aabbs = R.preprocess(bits)
        rec[f"codes{bits}"], rec[f"ids{bits}"], rec[f"aabbs{bits}"] = codes, ids, aabbs
        if codes.size > 1:
            bn, bb, root = oracle.ref_binary(1, bits, codes, aabbs)
            rec[f"lbvh{bits}_nodes"], rec[f"lbvh{bits}_bounds"] = bn, bb
            hn, hb, hroot = oracle.ref_binary(0, bits, codes, aabbs, 8)
            sets = sorted(sorted(s) for s in oracle.binary_leaf_sets(hn, hroot))
            flat = np.array([x for s in sets for x in [len(s)] + s], np.uint32)
            rec[f"hploc{bits}_leafsets"] = flat
    for method, tag in ((1, "lbvh"), (0, "hploc")):
        R.build(method, 8, 64)
        b = R.bvh()
        rec[f"{tag}_nodes"] = b["nodes"]
        rec[f"{tag}_prims"] = b["primitive_indices"]
        rec[f"{tag}_tris"] = b["triangles"]
        rec[f"{tag}_meta"] = np.array([b["root_reference"], b["internal_stack_bound"], b["packed_stack_bound"]],
                                      np.uint64)
        rec[f"{tag}_root_bounds"] = b["root_bounds"]
        if tag == "lbvh":
            rec["exact"] = R.exact(qx, qy, qz)
            for order in (0, 1, 2):
                rec[f"moment{order}"] = R.moments(order)
                rec[f"taylor{order}_b2"] = R.taylor(order, qx, qy, qz, 2.0)
                rec[f"taylor{order}_b1e6"] = R.taylor(order, qx, qy, qz, 1e6)
    rec["exact_f64"] = oracle.ref_exact_f64(mesh, qx, qy, qz)
    R.close()
    np.savez_compressed(OUT / f"{name}.npz", **rec)
    print(f"wrote {name}.npz")


def main() -> None:
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref/libgwnref.so is missing; build it with oracle/build.py where the "
                         "reference headers are present")
    OUT.mkdir(parents=True, exist_ok=True)
    for name, mesh in fixture_meshes().items():
        record(name, mesh)


if __name__ == "__main__":
    main()
