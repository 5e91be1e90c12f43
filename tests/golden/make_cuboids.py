"""Generates tests/golden/cuboids.npz from the upstream reference: uniformly
magnetised cuboid sources (SourceGeometry.UNIFORM_CUBOID).

Run where the reference's own pybind11 module has been built from its sources
(`make -f oracle/ref.mk`):

    python tests/golden/make_cuboids.py [--ref-module-dir oracle/_ref]

Fixtures (all seeded synthetic data):
  tensor__*   the cuboid -> point moment-to-field tensor, read off the
              reference's FP64 DenseDirectPlan as the fields of unit total
              moments along x, y, z (targets inside, on faces, edges and
              corners, at the centre, near and far);
  <case>__*   complete UniformFmm evaluations (CpuStatic, FP32 and FP64) with
              cuboid sources, common or per-source sizes, with and without
              the cuboid P2M, plus the FP64 dense direct sum of the same
              sources (H) and the reference's point-dipole potential; one
              case also keeps the FP32 per-node multipoles (cuboid P2M).
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(module_dir):
    sys.path.insert(0, module_dir)
    import cdfmm  # the upstream reference module

    return cdfmm


def sizes_list(ref, h):
    return [ref.CuboidSize(*map(float, row)) for row in np.atleast_2d(h)]


def tensor_case(ref, out, name, h, targets):
    src = np.zeros((1, 3))
    plan = ref.DenseDirectPlan(src, targets, source_geometry=ref.SourceGeometry.UNIFORM_CUBOID,
                               source_sizes=sizes_list(ref, h), static_precision="float64")
    cols = [np.asarray(plan.evaluate(np.eye(3)[[c]])) for c in range(3)]
    T = np.stack(cols, axis=-1)  # [target][field component][moment component]
    out[f"tensor__{name}__h"] = np.asarray(h, dtype=np.float64)
    out[f"tensor__{name}__targets"] = np.asarray(targets, dtype=np.float64)
    out[f"tensor__{name}__T"] = T


def fmm_case(ref, out, name, x, m, h, order, depth, cuboid_p2m, expansions=False):
    rec = {"sources": x, "moments": m, "sizes": np.atleast_2d(np.asarray(h, dtype=np.float64)),
           "order": np.int32(order), "depth": np.int32(depth), "cuboid_p2m": np.int32(cuboid_p2m)}
    for prec in (32, 64):
        o = ref.UniformFmmOptions()
        o.expansion_order = order
        o.tree.max_level = depth
        o.backend = ref.ExecutionBackend.CPU_STATIC
        o.precision = ref.StaticPrecision.FLOAT32 if prec == 32 else ref.StaticPrecision.FLOAT64
        o.source_geometry = ref.SourceGeometry.UNIFORM_CUBOID
        o.source_sizes = sizes_list(ref, h)
        o.use_cuboid_p2m = bool(cuboid_p2m)
        f = ref.UniformFmm(x, x, o)
        r = f.evaluate(m, output="both")
        rec[f"H{prec}"] = np.asarray(r["H"])
        rec[f"phi{prec}"] = np.asarray(r["phi"])
        if prec == 32 and expansions:
            nn = len(f.tree.nodes)
            rec["M32"] = np.stack([np.asarray(f.multipole(i)) for i in range(nn)])
    plan = ref.DenseDirectPlan(x, x, source_geometry=ref.SourceGeometry.UNIFORM_CUBOID,
                               source_sizes=sizes_list(ref, h), static_precision="float64")
    rec["H_direct"] = np.asarray(plan.evaluate(m))
    d = ref.direct_p2p_reference(x, x, m, "potential", list(range(len(x))))
    rec["phi_direct"] = np.asarray(d["phi"])
    for k, v in rec.items():
        out[f"{name}__{k}"] = v


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-module-dir", default=os.path.join(HERE, "..", "..", "oracle", "_ref"))
    args = ap.parse_args()
    ref = load_reference(os.path.abspath(args.ref_module_dir))
    out = {}
    rng = np.random.default_rng(61803)
    # ---- pair tensors --------------------------------------------------------
    for name, h in (("cube", (0.2, 0.2, 0.2)), ("slab", (0.4, 0.1, 0.05)), ("rod", (0.03, 0.05, 0.6))):
        hx, hy, hz = h
        special = [[0, 0, 0], [hx / 2, 0, 0], [0, -hy / 2, 0], [0, 0, hz / 2], [hx / 2, hy / 2, 0],
                   [hx / 2, -hy / 2, hz / 2], [0.3 * hx, 0.1 * hy, -0.4 * hz], [2 * hx, 0, 0], [0, 3 * hy, 0.5 * hz],
                   [1.5, -0.7, 2.0], [5.0, 5.0, 5.0]]
        near = rng.uniform(-1.5, 1.5, size=(40, 3)) * np.array(h)
        far = rng.normal(size=(20, 3)) * 2.0
        tensor_case(ref, out, name, h, np.concatenate([np.array(special, dtype=np.float64), near, far]))
    # ---- complete evaluations ---------------------------------------------------
    n = 3000
    x = rng.uniform(0.0, 1.0, size=(n, 3))
    m = rng.normal(size=(n, 3)) * 1e-3
    fmm_case(ref, out, "common_p6_d3", x, m, (0.03, 0.02, 0.025), 6, 3, 1, expansions=True)
    fmm_case(ref, out, "common_point_p2m_p6_d3", x, m, (0.03, 0.02, 0.025), 6, 3, 0)
    hs = rng.uniform(0.01, 0.05, size=(n, 3))
    fmm_case(ref, out, "per_source_p5_d3", x, m, hs, 5, 3, 1)
    # a lattice of touching cubes (a discretised magnet): the neighbours' own
    # near fields are the large, exact part
    g = (np.stack(np.meshgrid(*[np.arange(12)] * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) / 12.0
    mg = np.tile(np.array([[0.0, 0.0, 1.0]]), (len(g), 1)) / 12.0**3 + rng.normal(size=g.shape) * 1e-5
    fmm_case(ref, out, "touching_cubes_p6_d3", g, mg, (1 / 12, 1 / 12, 1 / 12), 6, 3, 1)
    np.savez_compressed(os.path.join(HERE, "cuboids.npz"), **out)
    print("cuboids.npz", os.path.getsize(os.path.join(HERE, "cuboids.npz")))


if __name__ == "__main__":
    main()
