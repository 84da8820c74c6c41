"""Shared checks of an aligner against the reference's known answers
(tests/golden/known_answers.json). `align(engine, q, t, qseed, tseed)` must return
(status, cigar, ed, qs, qe, ts, te)."""
import json
import os

from refgen import cigar_affine_cost, replay

ENGINES = {"wfa": 0, "affine": 1, "myers_fit": 2, "myers_global": 3}
HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


def _seq(case, key):
    if key in case:
        return case[key].encode()
    if key + "_repeat" in case:
        unit, n = case[key + "_repeat"]
        return unit.encode() * n
    n, base, muts = case[key + "_poly"]
    b = bytearray(base.encode() * n)
    for pos, ch in muts:
        b[pos] = ord(ch)
    return bytes(b)


def check_case(case, align):
    q, t = case["q"].encode(), case["t"].encode()
    r = align(ENGINES[case["engine"]], q, t, case.get("qseed", 0), case.get("tseed", 0))
    status, cigar, ed, qs, qe, ts, te = r
    src = case["src"]
    assert status == case.get("status", 0), (src, r)
    if status != 0:
        return
    if "ed" in case:
        assert ed == case["ed"], (src, r)
    if "cigar" in case:
        assert cigar == case["cigar"], (src, r)
    if "cigar_contains" in case:
        assert case["cigar_contains"] in cigar, (src, r)
    if "cigar_not_contains" in case:
        assert case["cigar_not_contains"] not in cigar, (src, r)
    if "ed_min" in case:
        assert ed >= case["ed_min"], (src, r)
    if "ed_max" in case:
        assert ed <= case["ed_max"], (src, r)
    for key, val in (("qs", qs), ("qe", qe), ("ts", ts), ("te", te)):
        if key in case:
            assert val == case[key], (src, key, r)
    if case.get("replay"):
        qseed, tseed = case.get("qseed", 0), case.get("tseed", 0)
        qi, ti = replay(cigar, q[qseed:], t[tseed:])
        assert qi == len(q) - qseed and ti == te - tseed, (src, r)
    if "indel_ops" in case:
        assert sum(1 for c in cigar if c in "ID") == case["indel_ops"], (src, r)
    if "affine_cost" in case:
        assert cigar_affine_cost(cigar, (2, 4, 1)) == case["affine_cost"], (src, r)


def check_pair(case, align):
    q, t = _seq(case, "q"), _seq(case, "t")
    ra = align(ENGINES[case["a"]], q, t, 0, 0)
    rb = align(ENGINES[case["b"]], q, t, 0, 0)
    idx = {"ed": 2, "cigar": 1, "te": 6}
    for f in case["fields"]:
        assert ra[idx[f]] == rb[idx[f]], (case["src"], f, ra, rb)
