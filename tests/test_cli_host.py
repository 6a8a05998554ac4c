"""CLI behaviour that is decided before any GPU work: flags, help/version, validation
messages and exit codes, and input-file parsing errors. Expected texts restate
xtneighbor_streaming/src/cli.cu:9-147 and src/util.cu:13-22."""
import os
import subprocess

import pytest

import xtn

pytestmark = pytest.mark.skipif(not os.path.exists(xtn.CLI_PATH), reason="CLI not built")


def run(args, cwd=None):
    p = subprocess.run([xtn.CLI_PATH] + args, capture_output=True, text=True, cwd=cwd)
    return p.returncode, p.stdout, p.stderr


def test_version_and_help():
    assert run(["-v"]) == (2, "2.0.0\n", "")
    rc, out, err = run(["--help"])
    assert rc == 2 and out.startswith("xt_neighbor: perform either nearest neighbor search") and err == ""
    assert "-N or --info-length [number] (required)" in out


@pytest.mark.parametrize(
    "args,msg",
    [
        (["-x"], "unknown option"),
        ([], "missing path for seq"),
        (["-i", "a.csv"], "missing length for seq"),
        (["-i", "a.csv", "-n", "0"], "invalid input length"),
        (["-i", "a.csv", "-n", "3", "-d", "0"], "distance must be a valid number larger than 0"),
        (["-i", "a.csv", "-n", "3", "-m", "cosine"], "invalid measure option"),
        (["-i", "a.csv", "-n", "3", "-I", "info.csv"], "repertiore path or repertoire count is missing in overlap mode"),
        (["-i", "a.csv", "-n", "3", "-N", "2"], "repertiore path or repertoire count is missing in overlap mode"),
        (["-i", "/nonexistent.csv", "-n", "3"], "input file reading failed"),
    ],
)
def test_argument_errors(args, msg):
    rc, out, err = run(args)
    assert rc == 1 and err == f"Error: {msg}\n"


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_input_errors(tmp_path):
    f = write(tmp_path, "a.csv", "cdr3\nCAAA\nCAXA\n")
    assert run(["-i", f, "-n", "2"])[2] == "Error: invalid char\nError: input parsing error\nError line: 3\n"
    f = write(tmp_path, "b.csv", "cdr3\nCAAA\nCADA\n")
    assert run(["-i", f, "-n", "3"])[2] == "Error: input length doesn't match with the actual\n"
    assert run(["-i", f, "-n", "1"])[2] == "Error: SeqArray exceeding max length\nError: input parsing error\nError line: 3\n"
    f = write(tmp_path, "c.csv", "cdr3\nCAAA\r\n")  # CRLF: '\r' is not a residue
    assert run(["-i", f, "-n", "1"])[2].startswith("Error: invalid char\n")


def test_overlap_input_errors(tmp_path):
    f = write(tmp_path, "s.csv", "cdr3,count\nCAAA,3\nCADA\n")
    i = write(tmp_path, "i.csv", "size\n2\n")
    rc, _, err = run(["-i", f, "-n", "2", "-I", i, "-N", "1"])
    assert rc == 1 and err == "Error: input parsing error (comma expected)\nError line: 3\n"
    f = write(tmp_path, "s2.csv", "cdr3,count\nCAAA,3\nCADA,0\n")
    assert run(["-i", f, "-n", "2", "-I", i, "-N", "1"])[2] == "Error: input parsing error (invalid number)\nError line: 3\n"
    i2 = write(tmp_path, "i2.csv", "size\n1\n")
    assert run(["-i", f, "-n", "2", "-I", i2, "-N", "1"])[2] == "Error: total repertoires' size does not match sequence count [2]\n"
    i3 = write(tmp_path, "i3.csv", "size\n1\n1\n")
    assert run(["-i", f, "-n", "2", "-I", i3, "-N", "1"])[2] == "Error: info length doesn't match with the actual\n"
    i4 = write(tmp_path, "i4.csv", "size\n3\n")
    assert run(["-i", f, "-n", "2", "-I", i4, "-N", "1"])[2] == "Error: total repertoires' size does not match sequence count [1]\n"


def test_airr_errors(tmp_path):
    f = write(tmp_path, "a.tsv", "sequence_id\tcdr3_aa\tduplicate_count\nA\tCAAA\t2\nB\tCAZA\t1\n")
    rc, _, err = run(["-a", "-i", f, "-n", "2"])
    assert rc == 1
    assert err == "Error: invalid char\nError: invalid seq\nError line: 1\nError: line parsing error\nError line: 1\n"
