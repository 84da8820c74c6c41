"""Oracle restatement of the variant-observation step of align_read (CPU only).

Known answers: detect_tandem_repeats' own tests (phraya-core/src/lib.rs, tests module),
the local-coverage window tests (phraya-align/src/local_coverage_tests.rs), and
hand-built alignments whose observations follow from extract_variants_from_cigar
(phraya-align/src/executor.rs:814-1046) by inspection.
"""
import math

import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200.batch import ALN_DTYPE, PackedReads, READ_RESULT_DTYPE


# (sequence, expected regions (start, end inclusive)) from lib.rs's tests.
REPEAT_CASES = [
    (b"ATATATATAT", [(0, 9)]),
    (b"CAGCAGCAGCAG", [(0, 11)]),
    (b"GATAGATAGATA", [(0, 11)]),
    (b"GCGCGCGC", [(0, 7)]),
    (b"AAAAAAAAA", [(0, 8)]),
    (b"ATGCATGATCGATCG", []),
    (b"A", []),
    (b"AT", []),
    (b"atatatatat", [(0, 9)]),
    (b"AtAtAtAtAt", [(0, 9)]),
    (b"CAGCAGCAGCAGCAGCAGCAG", [(0, 20)]),
    (b"CGGCGGCGGCGGCGGCGG", [(0, 17)]),
    (b"CTGCTGCTGCTGCTG", [(0, 14)]),
    (b"AGATAGATAGATAGATAGATAGAT", [(0, 23)]),
]


@pytest.mark.parametrize("seq,exp", REPEAT_CASES)
def test_tandem_repeats_known_answers(seq, exp):
    assert O.tandem_repeats(seq) == exp


def test_tandem_repeats_positional_cases():
    # detects_repeat_at_sequence_start / _end / _in_sequence_middle, multiple repeats
    assert any(s == 0 for s, _ in O.tandem_repeats(b"ATATATATATTGCAAA"))
    assert any(e == 14 for _, e in O.tandem_repeats(b"TGCAAATATATATAT"))
    mid = O.tandem_repeats(b"TGCAATATATATACCC")
    assert mid and all(5 >= s >= 3 for s, _ in mid)
    assert len(O.tandem_repeats(b"ATATATATAGCGCGCATATATAT")) >= 2
    assert len(O.tandem_repeats(b"ATATATATAGCGCGC")) >= 2
    # two AT units only: below min_repeat_count 3
    assert all((e - s + 1) >= 6 for s, e in O.tandem_repeats(b"ATATATGC"))


def test_tandem_repeats_walk_skips_accepted_repeat():
    # the walk jumps past an accepted repeat, so a later position inside it is never tested;
    # period 4 is tried before 3 and 2
    assert O.tandem_repeats(b"ACACACACAC" + b"GT") == [(0, 9)]  # ACAC twice only: period 2 wins
    assert O.tandem_repeats(b"ACGTACGTACGTAC") == [(0, 11)]
    assert O.tandem_repeats(b"GG" + b"TATATATA" + b"CCCCCCCCC") == [(2, 9), (10, 18)]
    assert O.tandem_repeats(b"AAAAAAAAAAAA") == [(0, 11)]
    assert O.tandem_repeats(b"AAAAAAAAAAAAAA") == [(0, 11)]


def _results(alns, reverse=0, has_result=1):
    """One read with the given alignments [(cigar, ed, ts, te)], primary first."""
    rr = np.zeros(1, dtype=READ_RESULT_DTYPE)
    rr["has_result"] = has_result
    rr["reverse"] = reverse
    rr["n_aln"] = len(alns)
    aln = np.zeros(max(len(alns), 1), dtype=ALN_DTYPE)
    cig = b""
    for i, (c, ed, ts, te) in enumerate(alns):
        aln[i]["edit_distance"] = ed
        aln[i]["target_start"] = ts
        aln[i]["target_end"] = te
        aln[i]["cigar_off"] = len(cig)
        aln[i]["cigar_len"] = len(c)
        cig += c
    return rr, aln, np.frombuffer(cig + b"\0", dtype=np.uint8).copy()


def _variants(target, read, alns, reverse=0, strategy=A.BALANCED, radius=0, hotspots=()):
    tg = O.Target(target)
    packed = PackedReads([read])
    rr, aln, cig = _results(alns, reverse)
    off, var, cov, al = tg.variants_packed(packed, rr, aln, cig, strategy, radius, hotspots)
    return O.unpack_variants(1, off, var, cov, al)[0]


TARGET = b"ACGTTGCAAGGCTTACGATCCGATGCAATGCCTAGGCATTACGGATCCAGTA"  # 52 bases


def test_snp_observation():
    read = bytearray(TARGET[10:30])
    read[5] = ord("A") if read[5] != ord("A") else ord("C")
    v = _variants(TARGET, bytes(read), [(b"5M1X14M", 1, 10, 30)], radius=4)
    assert len(v) == 1
    pos, ref, typ, rep, strand, ed, conf, kmer, cov, voff, alleles = v[0]
    assert (pos, ref, typ, strand, ed, kmer, voff) == (15, TARGET[15], 0, 0, 1, 1.0, 4)
    assert conf == 1.0 - 1 / 20
    assert cov == [1] * 9  # [11, 20): inside the single window [10, 30)
    assert alleles == [(read[5], 1)]


def test_deletion_and_insertion_observations():
    # I = target bases absent from the read (a deletion at t), D = read bases absent
    # from the target (an insertion at t, alleles = counted inserted bytes, ascending)
    read = TARGET[0:10] + TARGET[13:20] + b"GAG" + TARGET[20:30]
    v = _variants(TARGET, read, [(b"10M3I7M3D10M", 6, 0, 30)], radius=2)
    assert [(x[0], x[1], x[2]) for x in v] == [(10, TARGET[10], 2), (20, ord("."), 1)]
    assert v[0][10] == [(ord("."), 1)]
    assert v[1][10] == [(ord("A"), 1), (ord("G"), 2)]
    assert v[0][8] == [1, 1, 1, 1, 1] and v[0][9] == 2


def test_window_clipping_and_multi_alignment_coverage():
    read = bytes([ord("T") if TARGET[0] != ord("T") else ord("G")]) + TARGET[1:8]
    alns = [(b"1X7M", 1, 0, 8), (b"8M", 2, 4, 12), (b"8M", 2, 60, 68)]  # last window clipped away
    v = _variants(TARGET, read, alns, radius=6)
    assert len(v) == 1
    assert v[0][0] == 0 and v[0][9] == 0
    assert v[0][8] == [1, 1, 1, 1, 2, 2, 2]  # positions 0..6: [0,8) everywhere, [4,12) from 4
    # at the end of the target the window stops at target_len
    rd = TARGET[44:51] + bytes([ord("A") if TARGET[51] != ord("A") else ord("C")])
    v = _variants(TARGET, rd, [(b"7M1X", 1, 44, 52)], radius=5)
    assert v[0][0] == 51 and len(v[0][8]) == 6 and v[0][9] == 5


def test_hotspot_zeroes_kmer_uniqueness_and_confidence():
    read = bytearray(TARGET[10:30])
    read[0] = ord("A") if read[0] != ord("A") else ord("C")
    read[10] = ord("A") if read[10] != ord("A") else ord("C")
    v = _variants(TARGET, bytes(read), [(b"1X9M1X9M", 2, 10, 30)], hotspots=[(5, 11), (20, 21)])
    assert [x[7] for x in v] == [0.0, 0.0]
    assert [x[6] for x in v] == [0.0, 0.0]
    v = _variants(TARGET, bytes(read), [(b"1X9M1X9M", 2, 10, 30)], hotspots=[(5, 10), (21, 40)])
    assert [x[7] for x in v] == [1.0, 1.0]


def test_negative_score_gives_negative_zero_in_hotspot():
    # ed > |q|: primary_score < 0, and 0.0 * score is -0.0 as f64 arithmetic has it
    v = _variants(TARGET, b"AC", [(b"1X1X", 5, 0, 2)], hotspots=[(0, 2)])
    assert v[0][6] == 0.0 and math.copysign(1.0, v[0][6]) == -1.0


def test_reverse_strand_uses_reverse_complement():
    fwd = bytearray(TARGET[10:30])
    fwd[3] = ord("A") if fwd[3] != ord("A") else ord("C")
    rc = bytes(fwd[::-1]).translate(bytes.maketrans(b"ACGT", b"TGCA"))
    v = _variants(TARGET, rc, [(b"3M1X16M", 1, 10, 30)], reverse=1)
    assert v[0][4] == 1 and v[0][10] == [(fwd[3], 1)]


def test_strategy_radius_defaults():
    read = bytearray(TARGET[:52])
    read[26] = ord("A") if read[26] != ord("A") else ord("C")
    for strat, r in ((A.FAST, 150), (A.BALANCED, 50), (A.SENSITIVE, 25)):
        v = _variants(TARGET, bytes(read), [(b"26M1X25M", 1, 0, 52)], strategy=strat)
        assert len(v[0][8]) == min(26 + r + 1, 52) - max(0, 26 - r)


def test_repeat_flag_excludes_region_end():
    # is_in_repeat_region: pos < region.end with end inclusive, so the last base is outside
    target = b"GCTTGA" + b"CAG" * 4 + b"TTGACCTGA"  # CAG repeat at [6, 17]
    assert O.tandem_repeats(target) == [(6, 17)]
    read = bytearray(target)
    for p in (6, 16, 17):
        read[p] = ord("T")
    v = _variants(target, bytes(read), [(b"6M1X9M1X1X9M", 3, 0, len(target))])
    assert [(x[0], x[3]) for x in v] == [(6, 1), (16, 1), (17, 0)]


def _local_coverage_case(query, target):
    tg = O.Target(target)
    packed = PackedReads([query])
    rr, aln, cig, _ = tg.align_packed(packed, A.BALANCED, A.GAP_AFFINE, nthreads=1)
    off, var, cov, al = tg.variants_packed(packed, rr, aln, cig, A.BALANCED)
    return O.unpack_variants(1, off, var, cov, al)[0]


def test_reference_local_coverage_windows():
    # local_coverage_tests.rs: window sizes at the middle, start and end of the target
    base = b"ACGT" * 40
    t = bytearray(base)
    t[100] = ord("T")
    v = _local_coverage_case(base, bytes(t))
    mid = [x for x in v if x[0] == 100]
    assert mid and len(mid[0][8]) == 101
    q = b"TACT" + b"ACGT" * 36
    t = bytearray(q)
    t[0] = ord("A")
    v = _local_coverage_case(q, bytes(t))
    st = [x for x in v if x[0] == 0]
    assert st and len(st[0][8]) == 51
    t = bytearray(b"A" * 150)
    t[149] = ord("T")
    v = _local_coverage_case(b"A" * 150, bytes(t))
    en = [x for x in v if x[0] == 149]
    assert en and len(en[0][8]) == 51
    t = bytearray(b"ACGT" * 45)
    t[75] = ord("A")
    v = _local_coverage_case(b"ACGT" * 45, bytes(t))
    d = [x for x in v if x[0] == 75]
    assert d and len(d[0][8]) == 101 and all(c > 0 for c in d[0][8])


def test_coverage_merge_quantized_track_is_zero_and_depth_counts():
    # quantize_coverage(1) == ((1 + 2) / 5) * 5 == 0: per-read windows of count 1 merge to
    # an all-zero track, as merge_result builds it; the depth mode counts the windows
    aln = np.zeros(4, dtype=ALN_DTYPE)
    aln["target_start"] = [0, 5, 90, 200]
    aln["target_end"] = [10, 12, 120, 210]
    assert not O.coverage_merge(aln, 100).any()
    d = O.coverage_merge(aln, 100, depth=True)
    assert d[:14].tolist() == [1] * 5 + [2] * 5 + [1, 1, 0, 0]
    assert d[88:].tolist() == [0, 0] + [1] * 10
    assert int(d.sum()) == 10 + 7 + 10
