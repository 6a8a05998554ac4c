"""bench.py's roofline inputs, on the CPU: the algorithmic bytes of each kernel per step and the
ncu traffic read from the committed summaries."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

# counts of the 1M-sequence, d=2 workload
ST = {"n_variants": 109_554_745, "n_candidates": 5_557_204, "n_unique": 1_222_000, "id_bits": 20}


def test_algorithmic_bytes():
    n, nch = 1_000_000, 15_000_000
    V, P, U = ST["n_variants"], ST["n_candidates"], ST["n_unique"]
    assert bench.algorithmic_bytes("bucket_scatter", ST, n, nch) == 8.0 * V + 177.0 * n
    assert bench.algorithmic_bytes("bucket_split", ST, n, nch) == 16.0 * V
    assert bench.algorithmic_bytes("bucket_gen", ST, n, nch) == 8.0 * V + 177.0 * n
    assert bench.algorithmic_bytes("bucket_partition", ST, n, nch) == 16.0 * V
    assert bench.algorithmic_bytes("bucket_group", ST, n, nch) == 8.0 * V + 8.0 * P
    assert bench.algorithmic_bytes("pair_dedup", ST, n, nch) == 8.0 * P + 16.0 * U
    # 40-bit pair keys: five 8-bit passes over the distinct pairs
    assert bench.algorithmic_bytes("pair_sort_pass", ST, n, nch) == 16.0 * U * 5
    # without the hash set every candidate is verified
    no_set = dict(ST, n_unique=0)
    assert bench.algorithmic_bytes("verify", no_set, n, nch) > bench.algorithmic_bytes("verify", ST, n, nch)
    assert bench.algorithmic_bytes("no_such_kernel", ST, n, nch) is None


def test_traffic_comes_from_the_committed_summary():
    t = bench.ncu_traffic("bucket_scatter", "nn_1m_leven_d2")
    assert t is not None and t > 1e9  # dram read + write of one launch, bytes
    text = open(os.path.join(ROOT, "profiles", "bucket_scatter_nn_1m_leven_d2.md")).read()
    assert "ncu --set full --clock-control none" in text  # the command that made it
    assert bench.ncu_traffic("bucket_scatter", "no_such_workload") is None
