"""Shared pytest configuration.

Markers: `gpu` -- needs a CUDA device (B200); the CPU suite runs with
`-m "not gpu"`.  GPU tests are skipped only when no CUDA device exists at all;
a missing or unloadable library is an error, never a skip.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "dip-fmm_b200", "python")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


def pytest_collection_modifyitems(config, items):
    import cdfmm_b200

    if cdfmm_b200.device_count() > 0:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_group(filename, name):
    """Fields of one golden record stored as `<name>__<field>` in an npz."""
    data = np.load(os.path.join(GOLDEN, filename))
    prefix = name + "__"
    return {k[len(prefix):]: data[k] for k in data.files if k.startswith(prefix)}


def group_names(filename):
    data = np.load(os.path.join(GOLDEN, filename))
    return sorted({k.split("__")[0] for k in data.files})
