"""Generates tests/golden/pins.npz: golden vectors from the upstream reference
for the configurations the smaller fixtures (make_golden.py) do not reach.

Run in a container that has the reference sources, after
`make -f oracle/ref.mk REF=<reference checkout>` built its pybind11 module:

    python tests/golden/make_pins.py [--ref-module-dir oracle/_ref] [--cache DIR]

Cases (all seeded synthetic data; the reference runs its CpuStatic backend in
FP32 and FP64 and its FP64 direct sum):

  lattice_p8_d4   32^3 jittered lattice (spacing 1/32, jitter U(-0.1, 0.1)
                  spacings), N = 32,768, depth 4 (exactly 8 per leaf), p = 8,
                  one state of i.i.d. N(0, 1) moments (float32 values), field +
                  potential.  Inputs stored; outputs on a 4,096-target sample.
  uniform_p6_d5   N = 131,072 uniform in [0, 1)^3, depth 5 (~4 per leaf, the
                  far field dominates), p = 6, unit-direction x U[0.5, 1.5]
                  moments.  Positions regenerated from the seed and checked by
                  SHA-256; the reference tree's permutations and node ranges as
                  SHA-256 digests; outputs on a 4,096-target sample.
  small_p9_d3,    N = 4,096 uniform, depth 3, p = 9 and p = 10, unit moments;
  small_p10_d3    inputs and complete outputs stored.
  lattice_c2      the 64^3 jittered lattice of the batched split-precision
                  workload (N = 262,144, depth 5, p = 8), generated exactly as
                  bench.py's lattice leg does (seed 314159 + 11), its state 0:
                  reference FP64 CpuStatic and FP64 direct sum on the bench's
                  16,384-target sample (seed 314159 + 12).  Shows how much of the
                  split-BF16 result's error against the direct sum is the
                  p = 8 expansion's own truncation.
  clustered_6000  6,000 points in two Gaussian clusters (the dense-leaf
                  near-field test's geometry: up to ~7,500 near sources per
                  target), p = 5, depth 2, root (0.5, 0.5, 0.5) half-width 0.5;
                  for K = 1, 3, 8 the moment states that test draws, states 0
                  and K - 1: the reference's FP32 and FP64 CpuStatic fields, so
                  the test's bar rests on the reference's own FP32 error there.
  tree_c1         the reference tree of the uniform N = 1,048,576, depth 5
                  workload (bench.py seed 314159): SHA-256 of its permutations
                  and node ranges, so the host tree is pinned bit-exact at the
                  headline size.

Every input is regenerated by its consumer from the recipe here (the seeds
are in the case functions; tests/test_pins.py repeats them) and the fixture
keeps only the SHA-256 of the float64 input bytes, so a consumer that
regenerates different inputs fails on the digest instead of comparing against
the wrong fixture, and the fixture stays small.
"""

from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BENCH_SEED = 314159


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load_reference(module_dir):
    sys.path.insert(0, module_dir)
    import cdfmm  # the upstream reference module

    return cdfmm


def unit_moments(rng, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * rng.uniform(0.5, 1.5, size=(n, 1))


def jittered_lattice(rng, side):
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"), axis=-1).reshape(-1, 3)
    return (g + rng.uniform(-0.1, 0.1, size=g.shape)) / float(side)


def uniform_positions(seed, n):
    return np.random.default_rng(seed).uniform(0.0, 1.0, size=(n, 3))


def c2_lattice_inputs():
    """The bench's lattice leg inputs: positions and the K = 64 moment states."""
    rng = np.random.default_rng(BENCH_SEED + 11)
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64), np.arange(64), indexing="ij"), axis=-1).reshape(-1, 3)
    x = (g + rng.uniform(-0.1, 0.1, size=g.shape)) / 64.0
    m = rng.normal(size=(64, len(x), 3)).astype(np.float32)
    return x, m


def fmm_options(ref, order, depth, precision):
    o = ref.UniformFmmOptions()
    o.expansion_order = order
    o.tree.max_level = depth
    o.backend = ref.ExecutionBackend.CPU_STATIC
    o.precision = ref.StaticPrecision.FLOAT32 if precision == 32 else ref.StaticPrecision.FLOAT64
    return o


def tree_digests(ref, x, depth):
    o = ref.UniformTreeOptions()
    o.max_level = depth
    t = ref.UniformTree(x, x, o)
    ranges = np.array([(n.source_begin, n.source_end, n.target_begin, n.target_end) for n in t.nodes], dtype=np.int64)
    return dict(
        root=np.array([t.root_centre.x, t.root_centre.y, t.root_centre.z, t.root_half_width]),
        source_permutation_sha=sha(np.array(t.source_permutation, dtype=np.int32)),
        target_permutation_sha=sha(np.array(t.target_permutation, dtype=np.int32)),
        ranges_sha=sha(ranges),
        n_nodes=np.int64(len(ranges)),
    )


def evaluate(ref, x, m, order, depth, sample, precisions=(32, 64)):
    """Reference CpuStatic evaluations (targets = sources, self excluded) and
    the FP64 direct sum, all restricted to `sample`."""
    out = {}
    ids = list(range(len(x)))
    for prec in precisions:
        t0 = time.time()
        f = ref.UniformFmm(x, x, fmm_options(ref, order, depth, prec))
        r = f.evaluate(m, output="both", target_source_indices=ids)
        out[f"H{prec}"] = np.asarray(r["H"])[sample]
        out[f"phi{prec}"] = np.asarray(r["phi"])[sample]
        if prec == precisions[0]:
            st = f.static_plan_statistics
            out["transfer_classes"] = np.int64(st["transfer_classes"])
            out["interactions"] = np.int64(st["interactions"])
        print(f"    FP{prec} CpuStatic {time.time() - t0:.1f} s", flush=True)
        del f
    t0 = time.time()
    d = ref.direct_p2p_reference(x[sample], x, m, "both", list(map(int, sample)))
    out["H_direct"] = np.asarray(d["H"])
    out["phi_direct"] = np.asarray(d["phi"])
    print(f"    direct {time.time() - t0:.1f} s", flush=True)
    return out


def case_lattice_p8_d4(ref):
    rng = np.random.default_rng(8080)
    x = jittered_lattice(rng, 32)
    m = rng.normal(size=(len(x), 3)).astype(np.float32).astype(np.float64)
    sample = np.sort(np.random.default_rng(8081).choice(len(x), size=4096, replace=False)).astype(np.int64)
    rec = dict(sources=x, moments=m, order=np.int32(8), depth=np.int32(4), sample=sample)
    rec.update(evaluate(ref, x, m, 8, 4, sample))
    return rec


def case_uniform_p6_d5(ref):
    seed, n = 5150, 131072
    x = uniform_positions(seed, n)
    m = unit_moments(np.random.default_rng(seed + 1), n)
    sample = np.sort(np.random.default_rng(seed + 2).choice(n, size=4096, replace=False)).astype(np.int64)
    rec = dict(seed=np.int64(seed), n=np.int64(n), positions_sha=sha(x), moments_sha=sha(m), order=np.int32(6),
               depth=np.int32(5), sample=sample)
    rec.update({f"tree_{k}": v for k, v in tree_digests(ref, x, 5).items()})
    rec.update(evaluate(ref, x, m, 6, 5, sample))
    return rec


def case_small(ref, order):
    rng = np.random.default_rng(900 + order)
    x = rng.uniform(0.0, 1.0, size=(4096, 3))
    m = unit_moments(rng, 4096)
    sample = np.arange(4096, dtype=np.int64)
    rec = dict(sources=x, moments=m, order=np.int32(order), depth=np.int32(3), sample=sample)
    rec.update(evaluate(ref, x, m, order, 3, sample))
    return rec


def case_lattice_c2(ref):
    x, m = c2_lattice_inputs()
    n = len(x)
    sample = np.random.default_rng(BENCH_SEED + 12).choice(n, size=16384, replace=False).astype(np.int64)
    m0 = m[0].astype(np.float64)
    rec = dict(positions_sha=sha(x), moments_sha=sha(m0), order=np.int32(8), depth=np.int32(5), sample=sample)
    rec.update(evaluate(ref, x, m0, 8, 5, sample, precisions=(64,)))
    return rec


def clustered_6000(seed):
    """The dense-leaf test's geometry (tests/test_gpu_parity.py): 6,000 points
    in two Gaussian clusters (sigma 0.04) clipped into the unit cube."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.3, 0.7, (2, 3))
    x = np.clip(c[rng.integers(0, 2, 6000)] + rng.normal(scale=0.04, size=(6000, 3)), 0.001, 0.999)
    return rng, x


def case_clustered_6000(ref):
    rec = {}
    for K in (1, 3, 8):
        rng, x = clustered_6000(5)
        ms = rng.normal(size=(K, len(x), 3)).astype(np.float32)
        rec["sources"] = x
        for k in sorted({0, K - 1}):
            m = ms[k].astype(np.float64)
            res = {}
            for prec in (32, 64):
                o = fmm_options(ref, 5, 2, prec)
                o.tree.root_centre = ref.Vec3(0.5, 0.5, 0.5)
                o.tree.root_half_width = 0.5
                f = ref.UniformFmm(x, x, o)
                res[prec] = f.evaluate(m, output="both", target_source_indices=list(range(len(x))))
            h64, p64 = np.asarray(res[64]["H"]), np.asarray(res[64]["phi"])
            # the FP64 field as float32 (its rounding, 6e-8, is far below the
            # bars it is used with) and the reference FP32 error against it
            rec[f"K{K}_s{k}_H64"] = h64.astype(np.float32)
            rec[f"K{K}_s{k}_phi64"] = p64.astype(np.float32)
            rec[f"K{K}_s{k}_ref32_rel_l2_H"] = np.float64(rel_l2(np.asarray(res[32]["H"]), h64))
            rec[f"K{K}_s{k}_ref32_rel_l2_phi"] = np.float64(rel_l2(np.asarray(res[32]["phi"]), p64))
            rec[f"K{K}_s{k}_moments_sha"] = sha(ms[k])
    return rec


def case_tree_c1(ref):
    x = uniform_positions(BENCH_SEED, 1048576)
    rec = dict(seed=np.int64(BENCH_SEED), n=np.int64(len(x)), positions_sha=sha(x), depth=np.int32(5))
    rec.update({f"tree_{k}": v for k, v in tree_digests(ref, x, 5).items()})
    return rec


CASES = {
    "small_p9_d3": lambda ref: case_small(ref, 9),
    "small_p10_d3": lambda ref: case_small(ref, 10),
    "lattice_p8_d4": case_lattice_p8_d4,
    "uniform_p6_d5": case_uniform_p6_d5,
    "clustered_6000": case_clustered_6000,
    "tree_c1": case_tree_c1,
    "lattice_c2": case_lattice_c2,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-module-dir", default=os.path.join(HERE, "..", "..", "oracle", "_ref"))
    ap.add_argument("--cache", default=None, help="directory for per-case results (resume a partial run)")
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    ref = load_reference(os.path.abspath(args.ref_module_dir))
    recs = {}
    for name, fn in CASES.items():
        path = os.path.join(args.cache, name + ".npz") if args.cache else None
        if path and os.path.exists(path):
            recs[name] = dict(np.load(path))
            continue
        if args.only is not None and name not in args.only:
            continue
        print(name, flush=True)
        t0 = time.time()
        recs[name] = fn(ref)
        print(f"  {name}: {time.time() - t0:.1f} s", flush=True)
        if path:
            os.makedirs(args.cache, exist_ok=True)
            np.savez_compressed(path, **recs[name])
    if set(recs) == set(CASES):
        for rec in recs.values():
            for key in ("sources", "moments"):
                if key in rec:
                    rec[key + "_sha"] = sha(np.asarray(rec.pop(key), dtype=np.float64))
            # FP64 fields stored as float32: their rounding (6e-8 relative) is
            # far below every bar they are compared with (>= 3e-5)
            for key, v in rec.items():
                if isinstance(v, np.ndarray) and v.dtype == np.float64 and v.ndim >= 1 and key != "tree_root":
                    rec[key] = v.astype(np.float32)
        out = os.path.join(HERE, "pins.npz")
        np.savez_compressed(out, **{f"{k}__{f}": v for k, rec in recs.items() for f, v in rec.items()})
        print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()
