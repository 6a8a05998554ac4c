"""The CLI reads large inputs in parallel (file image cut at line starts, one thread per
segment); its outcome must be the sequential reader's. Restated here, the reference's reader
(xtneighbor_streaming/src/cli.cu:101-147, SeqArray::append src/codec.cu:175-196): fgets()
pieces of at most 499 characters (a longer line gives several rows), "\\n" and " \\n" skipped,
the row limit (-n) met before a row's own checks, the first failing piece in file order
decides the message and its line number. Files here are a few MB, so several threads run;
the cases put the failing row in late segments, next to long lines and blank lines.
Without a GPU a file that parses cleanly stops at the device ("no CUDA device"), which shows
the parse itself succeeded.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import xtn

pytestmark = pytest.mark.skipif(not os.path.exists(xtn.CLI_PATH), reason="CLI not built")

ALPHA = b"ACDEFGHIKLMNPQRSTVWY"
VALID = set(b"ACDEFGHIKLMNPQRSTVWY")


def ref_outcome(data: bytes, n: int, double: bool):
    """stderr of the reference's sequential reader, or None when the input parses."""
    pieces, i = [], 0
    while i < len(data):
        j = data.find(b"\n", i, i + 499)
        e = j + 1 if j >= 0 else min(len(data), i + 499)
        pieces.append(data[i:e])
        i = e
    line, count = 1, 0
    for p in pieces[1:]:
        line += 1
        s = p.split(b"\0")[0]
        if s in (b"\n", b" \n"):
            continue
        if count >= n:
            return f"Error: SeqArray exceeding max length\nError: input parsing error\nError line: {line}\n"
        k = 0
        while k < 500 and k < len(s):
            c = s[k]
            if c in b"\n,\t":
                break
            k += 1
            if c not in VALID:
                return f"Error: invalid char\nError: input parsing error\nError line: {line}\n"
        if k == 0:
            return f"Error: input parsing error\nError line: {line}\n"
        if double:
            if b"," not in s:
                return f"Error: input parsing error (comma expected)\nError line: {line}\n"
            m = re.match(rb"\s*([+-]?\d+)", s[s.index(b",") + 1 :])
            v = int(m.group(1)) if m else 0
            if v == 0 or v > 2**31 - 1 or v < -(2**31):
                return f"Error: input parsing error (invalid number)\nError line: {line}\n"
        count += 1
    if count != n:
        return "Error: input length doesn't match with the actual\n"
    return None


def rows(n, seed, double=False):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(8, 23))
        s = bytes(ALPHA[int(i)] for i in rng.integers(0, 20, L))
        out.append(s + (b",%d" % int(rng.integers(1, 1000)) if double else b""))
    return out


def run_cli(tmp_path, data: bytes, n: int, double: bool):
    f = tmp_path / "in.csv"
    f.write_bytes(data)
    args = [xtn.CLI_PATH, "-i", str(f), "-n", str(n)]
    if double:
        i = tmp_path / "info.csv"
        i.write_text(f"size\n{n}\n")
        args += ["-I", str(i), "-N", "1"]
    p = subprocess.run(args, capture_output=True, text=True, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    return p.returncode, p.stderr


def build(body_rows, double=False):
    return (b"cdr3,count\n" if double else b"cdr3\n") + b"\n".join(body_rows) + b"\n"


CASES = {
    "clean": lambda r: (r, 0),
    "bad_char_late": lambda r: (r[:150_000] + [b"CASXF"] + r[150_000:], 0),
    "empty_field": lambda r: (r[:80_000] + [b",5"] + r[80_000:], 0),
    "blank_lines": lambda r: (r[:10] + [b""] + r[10:90_000] + [b" "] + r[90_000:170_000] + [b""] + r[170_000:], 0),
    "limit_before_bad_char": lambda r: (r[:190_000] + [b"CAZF"] + r[190_000:], -80_000),
    "bad_char_before_limit": lambda r: (r[:50_000] + [b"CAZF"] + r[50_000:], -30_000),
    "long_line": lambda r: (r[:100_000] + [b"CAS" * 400] + r[100_000:], 0),
    "long_line_bad_tail": lambda r: (r[:120_000] + [b"C" * 700 + b"Z"] + r[120_000:], 0),
    "too_few_rows": lambda r: (r, 5),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_parallel_parse_matches_sequential_reader(tmp_path, case):
    body, dn = CASES[case](rows(200_000, seed=len(case)))
    data = build(body)
    assert len(data) > (2 << 20)
    n = len(body) + dn
    if case == "long_line":
        n += 2  # 1200 residues: three pieces, three rows
    exp = ref_outcome(data, n, False)
    rc, err = run_cli(tmp_path, data, n, False)
    if exp is None:
        assert rc == 1 and "no CUDA device" in err, err
    else:
        assert rc == 1 and err == exp


@pytest.mark.parametrize("where", ["none", "bad_number", "no_comma"])
def test_parallel_parse_two_columns(tmp_path, where):
    body = rows(160_000, seed=11, double=True)
    if where == "bad_number":
        body[140_001] = body[140_001].split(b",")[0] + b",0"
    elif where == "no_comma":
        body[99_999] = body[99_999].split(b",")[0]
    data = build(body, double=True)
    exp = ref_outcome(data, len(body), True)
    rc, err = run_cli(tmp_path, data, len(body), True)
    if exp is None:
        assert rc == 1 and "no CUDA device" in err, err
    else:
        assert rc == 1 and err == exp
