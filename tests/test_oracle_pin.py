"""The oracle restatement against the reference's own CPU test oracles.

Inputs are the reference tests' glibc rand() vectors (srand(2137));
expected outputs are the digests of the reference's test oracles
(tests/golden/ref_testoracles.json, made by tests/golden/make_golden.py from
oracle/_ref/libref_testoracles.so, compiled from the reference sources).
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import conftest as C
import oracle

GOLD = json.loads((Path(__file__).parent / "golden" / "ref_testoracles.json").read_text())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _inputs():
    v = {}
    for R in (20, 3, 10000):
        v[f"rle1_R{R}"] = lambda R=R: C.ref_rle1_input(R)
    for A in (256, 4, 1):
        v[f"bwt_A{A}"] = lambda A=A: C.ref_bwt_input(A)
    for A in (256, 4):
        v[f"mtf_A{A}"] = lambda A=A: C.ref_mtf_input(A)
    for R in (20, 10000):
        v[f"rle2_R{R}"] = lambda R=R: C.ref_rle2_input(R)
    v["rle2_incompressible"] = C.ref_rle2_incompressible
    return v


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_matches_reference_test_oracle(name):
    g = GOLD[name]
    a = _inputs()[name]()
    assert sha(a) == g["input_sha256"], "input generator drifted"
    st = g["stage"]
    if st == "rle1":
        out = oracle.rle1(a)
    elif st == "bwt":
        out = oracle.bwt(a)
    elif st == "mtf":
        # the reference test drives fmtf with SA[i] = (i+1) mod N so that the
        # last column is the input itself (tests/compression/fmtf.cu:13-19)
        sa = ((np.arange(a.size) + 1) % a.size).astype(np.int32)
        out, _, _, _ = oracle.mtf(a, sa)
    else:
        out = oracle.rle2(a, C.table_size(a))
    assert out.size == g["len"]
    assert sha(out) == g["output_sha256"]


def test_reference_testoracle_library_agrees_when_built():
    """If the reference's test oracles are built here, compare directly too."""
    R = oracle.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built on this machine")
    a = C.ref_bwt_input(4, 3000)
    ref = np.zeros(a.size, np.int32)
    R.ref_bwt(a.ctypes.data, a.size, ref.ctypes.data)
    assert np.array_equal(ref, oracle.bwt(a))
