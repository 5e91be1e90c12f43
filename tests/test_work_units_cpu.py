"""Host logic of the list-1 work units (no GPU): p2p_work_units cuts every
leaf's targets into units of at most 128 (fewer where a unit's cost --
targets x neighbourhood sources -- would pass total / (20 x SMs), 16 at
least), puts the units costing >= 4x the mean first, heaviest first, and
keeps the rest in Morton order.  A small C++ driver linked against the
library calls it on leaf offsets built here; the checks are that every
target is covered exactly once, the widths and the cap, the order, and that
a uniform geometry large enough for no leaf to reach the cap has exactly its
non-empty leaves as units, in Morton order.
"""

import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "dip-fmm_b200")
LIB_DIR = os.path.join(PKG, "lib")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "far_kernels.hpp"
int main() {
  int depth = 0, sms = 0, cap = 0;
  if (std::scanf("%d %d %d", &depth, &sms, &cap) != 3) return 2;
  const int leaves = 1 << (3 * depth);
  std::vector<int> so(static_cast<size_t>(leaves) + 1), to(static_cast<size_t>(leaves) + 1);
  for (int &v : so) if (std::scanf("%d", &v) != 1) return 2;
  for (int &v : to) if (std::scanf("%d", &v) != 1) return 2;
  for (const int4 &w : cdfmm_b200::p2p_work_units(so.data(), to.data(), depth, sms, cap != 0))
    std::printf("%d %d %d\n", w.x, w.y, w.z);
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++")
    lib = os.path.join(LIB_DIR, "libcdfmm_b200.so")
    if cxx is None or not os.path.exists(lib):
        pytest.skip("g++ or the built library is missing")
    d = tmp_path_factory.mktemp("units")
    src = d / "units.cpp"
    src.write_text(DRIVER)
    exe = d / "units"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(PKG, "csrc"), "-I", "/usr/local/cuda/include",
                    str(src), "-L", LIB_DIR, "-lcdfmm_b200", "-Wl,-rpath," + LIB_DIR, "-o", str(exe)],
                   check=True, capture_output=True)
    return str(exe)


def morton(ix, iy, iz):
    m = np.zeros_like(ix)
    for b in range(10):
        m |= ((ix >> b) & 1) << (3 * b)
        m |= ((iy >> b) & 1) << (3 * b + 1)
        m |= ((iz >> b) & 1) << (3 * b + 2)
    return m


def leaf_offsets(x, depth):
    side = 1 << depth
    c = np.clip(np.floor(x * side).astype(np.int64), 0, side - 1)
    counts = np.bincount(morton(c[:, 0], c[:, 1], c[:, 2]), minlength=side ** 3)
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def neighbourhood_sources(off, depth):
    """Sources in each leaf's clipped 3x3x3 neighbourhood, by Morton index."""
    side = 1 << depth
    z, y, x = np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij")
    m = morton(x, y, z)
    pad = np.pad(np.diff(off)[m], 1)  # [z][y][x]
    box = sum(pad[1 + dz:1 + dz + side, 1 + dy:1 + dy + side, 1 + dx:1 + dx + side]
              for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1))
    out = np.zeros(side ** 3, np.int64)
    out[m.ravel()] = box.ravel()
    return out


def run(driver, off, depth, sms, cap):
    text = f"{depth} {sms} {int(cap)}\n" + " ".join(map(str, off)) + "\n" + " ".join(map(str, off)) + "\n"
    out = subprocess.run([driver], input=text, capture_output=True, text=True, check=True).stdout
    return np.array([list(map(int, line.split())) for line in out.splitlines()], dtype=np.int64).reshape(-1, 3)


def clustered(rng, n):
    """n - n // 4 uniform points and a tight cluster (sigma 0.01) of n // 4."""
    c = rng.uniform(0.3, 0.7, 3)
    tight = np.clip(c + rng.normal(scale=0.01, size=(n // 4, 3)), 0.0, 0.999999)
    return np.concatenate([rng.uniform(0, 1, (n - n // 4, 3)), tight])


def test_uniform_geometry_units_are_its_leaves_in_morton_order(driver):
    # 400,000 points at depth 5 (~12 per leaf): the cap, total / (20 x 148),
    # is ~135 targets' worth of a leaf's neighbourhood, so no leaf is cut
    rng = np.random.default_rng(3)
    off = leaf_offsets(rng.uniform(0, 1, (400000, 3)), 5)
    units = run(driver, off, 5, 148, True)
    leaves = np.nonzero(np.diff(off))[0]
    np.testing.assert_array_equal(units[:, 0], leaves)
    np.testing.assert_array_equal(units[:, 1], off[leaves])
    np.testing.assert_array_equal(units[:, 2], np.diff(off)[leaves])


@pytest.mark.parametrize("cap", [False, True])
def test_clustered_units_cover_every_target_once_within_the_cap(driver, cap):
    rng = np.random.default_rng(11)
    depth, sms = 3, 148
    off = leaf_offsets(clustered(rng, 40000), depth)
    nt = np.diff(off)
    assert nt.max() > 5000
    units = run(driver, off, depth, sms, cap)
    leaf, t0, tn = units[:, 0], units[:, 1], units[:, 2]
    # exact cover, each unit inside its leaf
    order = np.argsort(t0)
    assert t0[order][0] == 0 and np.all(t0[order][1:] == (t0 + tn)[order][:-1]) and (t0 + tn).max() == off[-1]
    assert np.all(t0 >= off[leaf]) and np.all(t0 + tn <= off[leaf + 1])
    assert np.all((tn >= 1) & (tn <= 128))
    sources = neighbourhood_sources(off, depth)
    cost = tn * sources[leaf]
    total = int(np.sum(nt * sources))
    limit = max(1, total // (20 * sms))
    # every unit but a leaf's last has the leaf's full width
    last = t0 + tn == off[leaf + 1]
    if cap:
        fit = np.maximum(16, limit // np.maximum(sources[leaf], 1) // 16 * 16)
        width = np.where(128 * sources[leaf] > limit, fit, 128)
        assert np.all(tn[~last] == width[~last]) and np.all(tn <= width)
        assert np.all((cost <= limit) | (tn <= 16))
        assert len(units) > np.count_nonzero(nt) + (nt // 128).sum()  # the cap did cut
    else:
        assert np.all(tn[~last] == 128)
    # heavy units first, heaviest first; the rest in Morton order (with the
    # cap on, few units can reach 4x the mean)
    heavy = cost * len(units) >= 4 * total
    k = int(heavy.sum())
    assert k > 0 or cap
    assert np.all(heavy[:k]) and not np.any(heavy[k:])
    assert np.all(np.diff(cost[:k]) <= 0)
    rest = units[k:]
    assert np.all(np.diff(rest[:, 1]) > 0)
