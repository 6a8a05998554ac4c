"""Shared test setup: import paths, the `gpu` marker and small helpers.

Tests marked `gpu` need a CUDA device and call the product through its C ABI
(xt-neighbor_b200/lib/libxtn_b200.so). All other tests run on the CPU: the oracle
against the reference's own test vectors, the product's host/device helpers compiled for
the host, the CLI's argument and input handling, and the library's exported symbols.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "xt-neighbor_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the CUDA library")


def csr(seqs):
    import xtn

    return xtn.pack_sequences(seqs)


def assert_same_pairs(got_pairs, got_dist, exp_pairs, exp_dist, what=""):
    got_pairs = np.asarray(got_pairs, dtype=np.int32).reshape(-1, 2)
    exp_pairs = np.asarray(exp_pairs, dtype=np.int32).reshape(-1, 2)
    assert got_pairs.shape == exp_pairs.shape, f"{what}: {len(got_pairs)} pairs vs {len(exp_pairs)} expected"
    if len(exp_pairs):
        bad = np.nonzero((got_pairs != exp_pairs).any(axis=1))[0]
        assert len(bad) == 0, f"{what}: first differing row {bad[0]}: {got_pairs[bad[0]]} vs {exp_pairs[bad[0]]}"
    if exp_dist is not None:
        assert np.array_equal(np.asarray(got_dist, np.int8), np.asarray(exp_dist, np.int8)), f"{what}: distances differ"


@pytest.fixture(scope="session")
def kat():
    import json

    with open(os.path.join(GOLDEN, "reference_kat.json")) as f:
        return json.load(f)
