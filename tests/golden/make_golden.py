"""Generates the golden vectors under tests/golden/ from the upstream reference.

Run in a container that has the reference sources (it needs the reference's
own pybind11 module, built from those sources by `make -f oracle/ref.mk`):

    python tests/golden/make_golden.py [--ref-module-dir oracle/_ref]

Everything is seeded synthetic data.  The fixtures pin (a) the CPU oracle
(oracle/oracle.c) and (b) the B200 path: tree permutations, ranges and lists
(bit-exact), M2L class matrices, per-node FP32 expansions, and complete FP32 /
FP64 evaluations of the reference's CpuStatic backend plus its FP64 direct sum.
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


def unit_moments(rng, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * rng.uniform(0.5, 1.5, size=(n, 1))


def tree_case(ref, name, src, tgt, depth, root=None, out=None):
    o = ref.UniformTreeOptions()
    o.max_level = depth
    if root is not None:
        o.root_centre = ref.Vec3(*root[0])
        o.root_half_width = root[1]
    t = ref.UniformTree(src, tgt, o)
    nodes = t.nodes
    ranges = np.array([(n.source_begin, n.source_end, n.target_begin, n.target_end) for n in nodes], dtype=np.int64)
    out[name] = dict(
        sources=np.asarray(src, dtype=np.float64),
        targets=np.asarray(tgt, dtype=np.float64),
        depth=np.int32(depth),
        has_root=np.int32(root is not None),
        root_in=np.array(list(root[0]) + [root[1]] if root is not None else [0, 0, 0, 0], dtype=np.float64),
        root_centre=np.array([t.root_centre.x, t.root_centre.y, t.root_centre.z]),
        root_half_width=np.float64(t.root_half_width),
        source_permutation=np.array(t.source_permutation, dtype=np.int32),
        target_permutation=np.array(t.target_permutation, dtype=np.int32),
        ranges=ranges,
    )


def fmm_options(ref, order, depth, precision, root=None, fixed=None):
    o = ref.UniformFmmOptions()
    o.expansion_order = order
    o.tree.max_level = depth
    o.backend = ref.ExecutionBackend.CPU_STATIC
    o.precision = ref.StaticPrecision.FLOAT32 if precision == 32 else ref.StaticPrecision.FLOAT64
    if root is not None:
        o.tree.root_centre = ref.Vec3(*root[0])
        o.tree.root_half_width = root[1]
    if fixed is not None:
        o.fixed_target_source_indices = list(map(int, fixed))
    return o


def fmm_case(ref, name, src, tgt, moments, order, depth, ids, out, root=None, expansions=False):
    rec = dict(sources=src, targets=tgt, moments=moments, order=np.int32(order), depth=np.int32(depth),
               identities=np.asarray(ids if ids is not None else [], dtype=np.int32),
               has_root=np.int32(root is not None),
               root_in=np.array(list(root[0]) + [root[1]] if root is not None else [0, 0, 0, 0], dtype=np.float64))
    for prec in (32, 64):
        f = ref.UniformFmm(src, tgt, fmm_options(ref, order, depth, prec, root))
        r = f.evaluate(moments, output="both", target_source_indices=None if ids is None else list(map(int, ids)))
        rec[f"H{prec}"] = np.asarray(r["H"])
        rec[f"phi{prec}"] = np.asarray(r["phi"])
        if prec == 32:
            st = f.static_plan_statistics
            rec["transfer_classes"] = np.int64(st["transfer_classes"])
            rec["interactions"] = np.int64(st["interactions"])
            if expansions:
                nn = len(f.tree.nodes)
                rec["M32"] = np.stack([np.asarray(f.multipole(i)) for i in range(nn)])
                rec["L32"] = np.stack([np.asarray(f.local(i)) for i in range(nn)])
    d = ref.direct_p2p_reference(tgt, src, moments, "both", None if ids is None else list(map(int, ids)))
    rec["H_direct"] = np.asarray(d["H"])
    rec["phi_direct"] = np.asarray(d["phi"])
    out[name] = rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-module-dir", default=os.path.join(HERE, "..", "..", "oracle", "_ref"))
    args = ap.parse_args()
    ref = load_reference(os.path.abspath(args.ref_module_dir))

    # ---- tree parity -------------------------------------------------------
    trees = {}
    rng = np.random.default_rng(20240601)
    x = rng.uniform(0.0, 1.0, size=(4096, 3))
    tree_case(ref, "c0_uniform_d3", x, x, 3, out=trees)
    s = rng.uniform(-1.0, 2.0, size=(1500, 3))
    t = np.clip(rng.normal(0.5, 0.4, size=(1100, 3)), -1.0, 2.0)
    tree_case(ref, "separate_targets_d4", s, t, 4, out=trees)
    # points on the root faces, on internal boundaries and duplicated points
    b = np.array([[-1, -1, -1], [1, 1, 1], [0, 0, 0], [0.5, -0.5, 0.25], [1, -1, 0], [0, 0, 0],
                  [1 + 5e-13, 0, 0], [-0.25, 0.75, 1], [0.5, 0.5, 0.5], [0.5, 0.5, 0.5]], dtype=np.float64)
    tree_case(ref, "boundaries_explicit_root_d2", b, b[::-1].copy(), 2, root=((0.0, 0.0, 0.0), 1.0), out=trees)
    c = np.concatenate([rng.normal(0.2, 0.03, size=(300, 3)), rng.normal(0.8, 0.05, size=(200, 3))])
    tree_case(ref, "clusters_d5", c, c, 5, out=trees)
    tree_case(ref, "depth0", x[:50], x[:50], 0, out=trees)
    np.savez_compressed(os.path.join(HERE, "trees.npz"),
                        **{f"{k}__{f}": v for k, rec in trees.items() for f, v in rec.items()})

    # ---- interaction lists (geometry independent) ---------------------------
    lists = {}
    for depth in (2, 3):
        o = ref.UniformTreeOptions()
        o.max_level = depth
        t = ref.UniformTree([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]], o)
        l1 = [list(n.list1) for n in t.nodes]
        l2 = [list(n.list2) for n in t.nodes]
        lists[f"d{depth}__l1_off"] = np.cumsum([0] + [len(v) for v in l1]).astype(np.int32)
        lists[f"d{depth}__l1"] = np.array([i for v in l1 for i in v], dtype=np.int32)
        lists[f"d{depth}__l2_off"] = np.cumsum([0] + [len(v) for v in l2]).astype(np.int32)
        lists[f"d{depth}__l2"] = np.array([i for v in l2 for i in v], dtype=np.int32)
    np.savez_compressed(os.path.join(HERE, "lists.npz"), **lists)

    # ---- M2L class matrices --------------------------------------------------
    mats = {}
    offsets = [(2, 0, 0), (-3, 1, 2), (2, 2, -2), (3, 3, 3), (0, -2, 1), (-2, -3, 0)]
    for order in (2, 4, 6, 8):
        for o3 in offsets:
            key = f"p{order}__{o3[0]}_{o3[1]}_{o3[2]}"
            mats[key] = np.asarray(ref.static_m2l_matrix([0.0, 0.0, 0.0], list(map(float, o3)), order))
    # a non-integer, physical-scale translation as well
    mats["p6__phys"] = np.asarray(ref.static_m2l_matrix([0.1, -0.2, 0.05], [0.55, 0.3, -0.4], 6))
    np.savez_compressed(os.path.join(HERE, "m2l_matrices.npz"), **mats)

    # ---- complete evaluations -------------------------------------------------
    fmms = {}
    rng = np.random.default_rng(314159)
    x = rng.uniform(0.0, 1.0, size=(4096, 3))
    m = unit_moments(rng, 4096)
    fmm_case(ref, "c0", x, x, m, 4, 3, np.arange(4096), fmms)
    for order, depth in ((2, 2), (4, 3), (6, 4)):
        r2 = np.random.default_rng(9281 + order)
        x2 = r2.uniform(-0.9, 0.9, size=(48, 3))
        m2 = r2.normal(size=(48, 3))
        fmm_case(ref, f"small_p{order}_d{depth}", x2, x2, m2, order, depth, np.arange(48), fmms)
    r3 = np.random.default_rng(1701)
    xs = r3.uniform(0, 1, size=(700, 3))
    xt = r3.uniform(0.1, 0.9, size=(500, 3))
    ms = r3.normal(size=(700, 3))
    ids = np.full(500, -1, dtype=np.int32)
    ids[::3] = r3.integers(0, 700, size=len(ids[::3]))
    xt[::3] = xs[ids[::3]]  # those targets coincide with their identified source
    fmm_case(ref, "targets_partial_ids", xs, xt, ms, 5, 3, ids, fmms)
    r4 = np.random.default_rng(741)
    x4 = r4.uniform(-1, 1, size=(600, 3))
    m4 = unit_moments(r4, 600)
    fmm_case(ref, "expansions_p4_d3", x4, x4, m4, 4, 3, np.arange(600), fmms, expansions=True)
    fmm_case(ref, "depth0", x4[:200], x4[:200], m4[:200], 3, 0, np.arange(200), fmms)
    r5 = np.random.default_rng(42)
    x5 = r5.uniform(-2, 3, size=(3000, 3))
    m5 = unit_moments(r5, 3000)
    fmm_case(ref, "p6_d4_explicit_root", x5, x5, m5, 6, 4, np.arange(3000), fmms, root=((0.5, 0.5, 0.5), 2.6))
    np.savez_compressed(os.path.join(HERE, "fmm.npz"),
                        **{f"{k}__{f}": v for k, rec in fmms.items() for f, v in rec.items()})
    for f in ("trees.npz", "lists.npz", "m2l_matrices.npz", "fmm.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
