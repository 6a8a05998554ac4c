"""Byte-for-byte parity with the reference binary on the benchmark's full-size workloads.

The reference XTNeighbor-streaming CLI (built from its sources by oracle/build_ref.sh into
oracle/_ref/xt_neighbor_ref) and this build's xt_neighbor run on the same files, written by
the generator command (bin/xtn_synth) with the benchmark's seeds, with -o; the output files
must be identical:
  * 10,000,000 sequences (clusters), Levenshtein d = 2 and Hamming d = 2;
  * 64 repertoires (23.9M rows, log-uniform sizes 1e4..2e6, shared pool), overlap, d = 1.
The reference needs about 100 s per 10M search on a B200. Its output lengths are the
benchmark's expect_out values. Skipped where the reference build is absent.
"""
import filecmp
import os
import subprocess

import pytest

import bench
import oracle as orc
import xtn

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(orc.REF_CLI), reason="reference build absent")]


def run_both_to_files(tmp_path, args):
    paths = []
    for name, exe in (("ours", xtn.CLI_PATH), ("ref", orc.REF_CLI)):
        out = tmp_path / f"{name}.txt"
        p = subprocess.run([exe] + args + ["-o", str(out)], capture_output=True, text=True, timeout=1800,
                           env=dict(os.environ, LC_ALL="C"))
        assert p.returncode == 0, f"{name}: rc={p.returncode} {p.stderr[-500:]}"
        paths.append(out)
    return paths


def line_count(path):
    with open(path, "rb") as f:
        return sum(chunk.count(b"\n") for chunk in iter(lambda: f.read(1 << 24), b""))


@pytest.mark.parametrize("workload", ["nn_10m_leven_d2", "nn_10m_hamming_d2"])
def test_10m_output_identical(tmp_path, workload):
    w = bench.WORKLOADS[workload]
    args = bench.workload_files(str(tmp_path), w)
    ours, ref = run_both_to_files(tmp_path, args)
    assert os.path.getsize(ours) == os.path.getsize(ref)
    assert filecmp.cmp(ours, ref, shallow=False), f"{workload}: output files differ"
    assert line_count(ref) == w["expect_out"]


def test_64_repertoire_overlap_identical(tmp_path):
    w = bench.WORKLOADS["overlap_64rep_leven_d1"]
    args = bench.workload_files(str(tmp_path), w)
    assert int(args[args.index("-n") + 1]) > 20_000_000
    ours, ref = run_both_to_files(tmp_path, args)
    assert filecmp.cmp(ours, ref, shallow=False), "overlap output files differ"
    assert line_count(ref) > 1000
