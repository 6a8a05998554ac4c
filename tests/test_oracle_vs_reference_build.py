"""The oracle's codec and deletion-variant generator against the reference's own code.

oracle/build_ref.sh compiles a host harness around the reference's expand_keys(),
str_encode(), len_decode() and remove_char() (xtneighbor_streaming/src/codec.cu,
generate_combination.cu; host-callable under TEST_ENV). This test feeds it random
sequences and distances 1..5 and requires the oracle to produce the same words in the
same order. Skipped where the harness was not built (it needs the reference sources).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.skipif(not os.path.exists(orc.REF_HARNESS), reason="reference harness not built")


def run_harness(cases):
    inp = "".join(f"{s} {d}\n" for s, d in cases)
    out = subprocess.run([orc.REF_HARNESS], input=inp, capture_output=True, text=True, check=True).stdout
    lines = out.splitlines()
    res, i = [], 0
    for _ in cases:
        e = lines[i].split()
        assert e[0] == "E"
        enc = [int(x) for x in e[1:4]]
        ln = int(e[4])
        i += 1
        rem = []
        while lines[i].startswith("R "):
            rem.append([int(x) for x in lines[i].split()[2:5]])
            i += 1
        v = lines[i].split()
        assert v[0] == "V"
        cnt = int(v[1])
        i += 1
        var = [[int(x) for x in lines[i + k].split()] for k in range(cnt)]
        i += cnt
        res.append((enc, ln, rem, var))
    return res


def test_codec_and_variants_match_reference():
    rng = np.random.default_rng(11)
    alpha = "ACDEFGHIKLMNPQRSTVWY"
    cases = []
    for _ in range(400):
        L = int(rng.integers(1, 26))
        # small alphabets give runs of equal residues (duplicate variants)
        sub = alpha[: int(rng.integers(2, 21))]
        s = "".join(rng.choice(list(sub), L))
        d = int(rng.integers(1, 6)) if L <= 14 else int(rng.integers(1, 4))
        cases.append((s, d))
    ref = run_harness(cases)
    for (s, d), (enc, ln, rem, var) in zip(cases, ref):
        w = orc.str_encode(s)
        assert list(w) == enc, s
        assert orc.len_decode(w) == ln, s
        for p, r in enumerate(rem):
            assert list(orc.remove_char(w, p)) == r, (s, p)
        assert orc.expand_words(s, d).tolist() == var, (s, d)
