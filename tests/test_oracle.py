"""Pins the CPU oracle to phraya's own known answers and seeded property sweeps.

The reference (Rust) cannot be built here, so the oracle's parity is established by
replaying the reference's test fixtures: literal known answers (golden JSON with
file:line) and the seeded generators of its property tests, checked with independent
O(nm) DP / Gotoh oracles exactly as the reference's tests do.
"""
import pytest

import oracle as O
from phraya_b200 import _abi as A
import known
import refgen as R


def oracle_align(engine, q, t, qseed, tseed):
    return O.extend(engine, [(q, t, qseed, tseed)], nthreads=1)[0]


KA = known.load()


@pytest.mark.parametrize("case", KA["cases"], ids=[c["src"] for c in KA["cases"]])
def test_known_answer(case):
    known.check_case(case, oracle_align)


@pytest.mark.parametrize("case", KA["pairs_equal"], ids=[c["src"] for c in KA["pairs_equal"]])
def test_engines_agree_where_reference_asserts(case):
    known.check_pair(case, oracle_align)


def test_lcp_battery_matches_scalar():
    # wfa_simd.rs:3857-3890: every LCP tier equals the byte-by-byte scalar reference.
    for a, b in R.lcp_battery():
        n = min(len(a), len(b))
        i = 0
        while i < n and a[i] == b[i]:
            i += 1
        assert O.lcp(a, b) == i
    assert O.lcp(b"ACGTACGT", b"ACGTTCGT") == 4  # wfa_simd.rs:3821-3826


def test_linear_global_edit_distance_matches_scalar_dp():
    # edit_distance_matches_scalar_property (wfa_simd.rs:3028-3051), 320 seeded cases.
    cases = R.scalar_edit_sweep()
    res = O.extend(A.ENGINE_WFA_LINEAR, cases)
    mye = O.extend(A.ENGINE_MYERS_GLOBAL, cases)
    for (q, t), r, m in zip(cases, res, mye):
        exp = R.edit_distance_dp(q, t)
        assert r[2] == exp, (q, t, r)
        assert m[2] == exp, (q, t, m)
        if q or t:
            qi, ti = R.replay(r[1], q, t)
            assert (qi, ti) == (len(q), len(t))
            qi, ti = R.replay(m[1], q, t)
            assert (qi, ti) == (len(q), len(t))
            assert R.levenshtein_from_cigar(r[1]) == exp


def test_affine_fitting_matches_gotoh():
    # affine_score_matches_gotoh_oracle_across_random_cases (wfa_simd.rs:3314-3371).
    cases = R.affine_fitting_cases()
    res = O.extend(A.ENGINE_WFA_AFFINE, cases)
    checked = 0
    for (q, t), r in zip(cases, res):
        if r[0] != 0:
            continue
        qi, ti = R.replay(r[1], q, t)
        assert qi == len(q) and ti == r[6]
        assert R.cigar_affine_cost(r[1], (2, 4, 1)) == R.gotoh(q, t, (2, 4, 1), True), (q, t, r)
        assert r[2] == R.levenshtein_from_cigar(r[1])
        checked += 1
    assert checked > 40


def test_affine_global_matches_gotoh():
    # affine_score_matches_gotoh_oracle_in_global_mode (wfa_simd.rs:3401-3454).
    cases = R.affine_global_cases()
    res = O.extend(A.ENGINE_WFA_AFFINE, cases)
    checked = 0
    for (q, t), r in zip(cases, res):
        assert len(t) <= len(q) + len(q) // 2 + 10
        if r[0] != 0:
            continue
        assert r[6] == len(t)
        qi, ti = R.replay(r[1], q, t)
        assert (qi, ti) == (len(q), len(t))
        assert R.cigar_affine_cost(r[1], (2, 4, 1)) == R.gotoh(q, t, (2, 4, 1), False), (q, t, r)
        checked += 1
    assert checked > 25


def test_myers_fitting_matches_wfa_sweep():
    # issue_176_myers_fitting_edit_distance_matches_wfa_sweep (test_wfa_algorithm.rs:375-436).
    cases = R.myers_wfa_fitting_sweep()
    assert len(cases) >= 300
    my = O.extend(A.ENGINE_MYERS_FIT, cases)
    wf = O.extend(A.ENGINE_WFA_LINEAR, cases)
    for (q, t), a, b in zip(cases, my, wf):
        assert a[0] == 0 and b[0] == 0
        assert a[2] == b[2], (q, t, a, b)
        for r in (a, b):
            qi, ti = R.replay(r[1], q, t)
            assert qi == len(q) and ti == r[6]


def test_seed_beyond_end_is_invalid_input():
    # lib.rs:322-346 (myers_extend) and :145-149 (wfa_extend_affine).
    assert O.myers_extend(b"ACGT", b"ACGTACGT", 5, 0)[0] == A.PHR_INVALID_INPUT
    assert O.myers_extend(b"ACGT", b"ACGT", 0, 10)[0] == A.PHR_INVALID_INPUT
    assert O.wfa_extend_affine(b"ACGT", b"ACGT", 0, 10)[0] == A.PHR_INVALID_INPUT


def test_empty_edges():
    # wfa_simd.rs:194-203 (both empty), :365-367 (empty query), :593-601 (affine qn==0),
    # :3793-3798 (Myers fitting m==0 / n==0).
    assert O.wfa_extend(b"", b"") == (0, "", 0, 0, 0, 0, 0)
    assert O.wfa_extend(b"", b"ACGT") == (0, "", 0, 0, 0, 0, 0)
    assert O.wfa_extend(b"ACG", b"") == (0, "3D", 3, 0, 3, 0, 0)
    assert O.wfa_extend_affine(b"", b"ACGT") == (0, "", 0, 0, 0, 0, 0)
    assert O.myers_extend(b"", b"ACGT") == (0, "", 0, 0, 0, 0, 0)
    assert O.myers_extend(b"ACGT", b"") == (0, "4D", 4, 0, 4, 0, 0)


# ---------------------------------------------------------------------------
# score_alignments (phraya-align/src/lib.rs:205-320)
# ---------------------------------------------------------------------------
def test_score_alignments_reference_cases():
    p = ("100M", 2, 0, 100, 0, 100)
    pi, alts = O.score_alignments([("100M", 0, 0, 100, 0, 100)], 100)
    assert (pi, alts) == (0, [])
    assert O.score_alignments([p, ("98M1I1D", 3, 0, 100, 0, 100)], 100) == (0, [1])
    assert O.score_alignments([p, ("80M10I10D", 20, 0, 100, 0, 100)], 100) == (0, [])
    assert O.score_alignments([("10M", 1, 0, 10, 0, 10), ("9M1D", 1, 0, 10, 0, 10)], 10) == (0, [1])
    assert O.score_alignments([("100M", 1, 0, 100, 0, 100), ("99M1D", 1, 0, 100, 0, 100)], 100) == (0, [1])
    with pytest.raises(ValueError):
        O.score_alignments([], 100)
    # primary = FIRST minimum; exact duplicates of the primary are not alternatives
    assert O.score_alignments([("5M", 1, 0, 5, 0, 5), ("5M", 0, 0, 5, 0, 5), ("5M", 0, 0, 5, 0, 5)], 5) == (1, [])


# ---------------------------------------------------------------------------
# Seeding (phraya-align/src/seeding.rs:113-170)
# ---------------------------------------------------------------------------
def test_seeding_cap_masks_hyperfrequent_minimizer():
    tv = [7, 7, 7, 7, 7, 9]
    tp = [10, 20, 30, 40, 50, 100]
    seeds = O.find_seeds(tv, tp, [7, 9], [0, 5], 2**64 - 1)
    assert len(seeds) == 6
    capped = O.find_seeds(tv, tp, [7, 9], [0, 5], 4)
    assert len(capped) == 1 and capped[0][2] == 9


def test_occurrence_cap_cases():
    assert O.occurrence_cap(list(range(1000)), list(range(1000))) == 256
    v = list(range(999)) + [9999] * 10000
    assert O.occurrence_cap(v, [0] * len(v)) == 256
    v = [x for x in range(500) for _ in range(100)]
    assert O.occurrence_cap(v, [0] * len(v)) == 800
    assert O.occurrence_cap([], []) == 256


def test_seeds_sorted_stably_by_query_pos():
    # find_seeds_indexed_capped emits in query-sketch order then stable-sorts by qpos.
    seeds = O.find_seeds([1, 2, 1], [50, 60, 70], [2, 1], [9, 3], 1000)
    assert seeds == [(3, 50, 1), (3, 70, 1), (9, 60, 2)]


# ---------------------------------------------------------------------------
# Chaining (phraya-align/src/chaining.rs:246-345)
# ---------------------------------------------------------------------------
def diagonal_seeds(target_start, query_start, count, spacing):
    return [(query_start + i * spacing, target_start + query_start + i * spacing, 0x1000 + i) for i in range(count)]


def test_chaining_reference_cases():
    assert O.chain_seeds([]) == []
    assert O.chain_seeds([(0, 1000, 1)], min_chain_score=25) == []
    ch = O.chain_seeds([(0, 1000, 1)], min_chain_score=10)
    assert len(ch) == 1 and len(ch[0][2]) == 1 and ch[0][1] == 1000
    ch = O.chain_seeds(diagonal_seeds(1000, 0, 5, 40))
    assert len(ch) == 1 and len(ch[0][2]) == 5 and ch[0][1] == 1000
    ch = O.chain_seeds(diagonal_seeds(1000, 0, 3, 40) + diagonal_seeds(1005, 160, 3, 40))
    assert len(ch) == 1 and len(ch[0][2]) == 6
    ch = O.chain_seeds(diagonal_seeds(1000, 0, 4, 40) + diagonal_seeds(6000, 0, 4, 40))
    assert len(ch) == 2 and {c[1] for c in ch} == {1000, 6000}
    ch = O.chain_seeds(diagonal_seeds(1000, 0, 6, 40) + [(500, 9000, 0xDEAD)])
    assert len(ch[0][2]) == 6 and ch[0][1] == 1000
    ch = O.chain_seeds([(0, 1000, 1), (40, 1240, 2)], min_chain_score=10)
    assert len(ch) == 2


def test_anchor_target_start_projection():
    # Chain::target_start = max(t0 - q0, 0) (chaining.rs:32-35)
    ch = O.chain_seeds([(30, 20, 1)], min_chain_score=10)
    assert ch[0][1] == 0


# ---------------------------------------------------------------------------
# Sketcher (this project's documented scheme, shared with the CUDA sketcher)
# ---------------------------------------------------------------------------
def test_sketch_density_and_strand_symmetry():
    seq = R.diverse_dna(5000, 11)
    v, p = O.sketch(seq)
    assert 0.12 < len(v) / 5000 < 0.22  # ~2/(w+1)
    assert all(p[i] < p[i + 1] for i in range(len(p) - 1))
    rc = seq[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    rv, rp = O.sketch(rc)
    common = len(set(v.tolist()) & set(rv.tolist()))
    assert common / len(set(v.tolist())) > 0.95
    # protein path: plain minimizers over bytes
    pv, pp = O.sketch(b"MKTAYIAKQRQISFVKSHFSRQLEERLGLIEVQ", 6, 5, A.ALPHABET_PROTEIN)
    assert len(pv) > 0
    assert O.sketch(b"ACGT")[0].size == 0  # shorter than k


# ---------------------------------------------------------------------------
# align_read (executor.rs:1333-1438, chaining_correctness.rs:41-154)
# ---------------------------------------------------------------------------
def revcomp(s):
    return s[::-1].translate(bytes.maketrans(b"ACGTacgt", b"TGCAtgca"))


def test_align_read_clean_snp_all_strategies():
    target = R.diverse_dna(300, 1)
    read = bytearray(target[50:200])
    read[30] = ord("C") if read[30] == ord("A") else ord("A")
    tg = O.Target(target)
    for strat in (A.FAST, A.BALANCED, A.SENSITIVE):
        (res,), _ = tg.align_reads([bytes(read)], strategy=strat)
        outcome, has, rev, alns = res
        assert has and not rev
        cigar, ed, qs, qe, ts, te = alns[0]
        assert ed == 1 and ts == 50
        # the single X lies at target position 80
        pos = ts
        xs = []
        for n, op in R.cigar_ops(cigar):
            if op == "X":
                xs.append(pos)
            if op in "MXI":
                pos += n
        assert xs == [80], (strat, cigar)


def test_align_read_indel_and_multimap():
    target = R.diverse_dna(300, 2)
    read = bytearray(target[50:200])
    del read[60]
    tg = O.Target(target)
    for strat in (A.BALANCED, A.SENSITIVE):
        (res,), _ = tg.align_reads([bytes(read)], strategy=strat)
        assert res[1] and "I" in res[3][0][0]  # target-extra base = reference deletion
    unit = R.diverse_dna(200, 3)
    target = unit + R.diverse_dna(500, 4) + unit + R.diverse_dna(500, 6)
    tg = O.Target(target)
    (res,), _ = tg.align_reads([unit[20:170]], strategy=A.SENSITIVE)
    assert res[1] and len(res[3]) >= 2
    tg = O.Target(R.diverse_dna(300, 5))
    tg.align_reads([R.diverse_dna(150, 999)], strategy=A.BALANCED)  # must not crash


def test_align_read_reverse_strand_and_stats():
    target = R.diverse_dna(300, 7)
    region = bytearray(target[100:200])
    region[50] = ord("C") if region[50] == ord("A") else ord("A")
    tg = O.Target(target)
    (res,), _ = tg.align_reads([revcomp(bytes(region))], strategy=A.BALANCED)
    assert res[1] and res[2] == 1
    assert abs(res[3][0][4] - 100) <= 1
    target = R.diverse_dna(300, 3)
    tg = O.Target(target)
    div = bytearray(target[50:200])
    for i in range(67, 82):
        div[i] = ord("C") if div[i] == ord("A") else ord("A")
    _, st = tg.align_reads([target[50:150], bytes(div), R.diverse_dna(120, 987654)], strategy=A.BALANCED)
    placed, no_seed, below, fast, none = st
    assert (placed, no_seed, below) == (1, 1, 1)


def test_align_read_stored_empty_sketch_is_no_seed():
    # executor.rs:671-674: an empty stored sketch with no seeds -> None / NoSeed
    target = R.diverse_dna(300, 3)
    tg = O.Target(target)
    e = (__import__("numpy").zeros(0, "u8"), __import__("numpy").zeros(0, "u4"))
    (res,), st = tg.align_reads([target[50:150]], stored=[e])
    assert res[0] == A.OUT_NO_SEED and res[1] == 0


def test_protein_wfa_and_myers_agree():
    # protein_wfa_myers_edit_distance_agree (phraya-align/src/executor.rs:2001-2027):
    # both engines compare raw bytes, so their distances agree on protein too
    for q, t in R.protein_wfa_myers_cases():
        w = O.wfa_extend(q, t)
        m = O.myers_extend(q, t)
        assert w[0] == 0 and m[0] == 0
        assert w[2] == m[2], (q, t, w, m)


def test_protein_alignment_never_reverse():
    # protein_alignment_never_attempts_reverse_strand (executor.rs:1965-1995): a protein
    # read with one substitution against its source region aligns forward, and its
    # variant observations say so
    target = R.diverse_protein(300, 11)
    region = bytearray(target[100:200])
    region[50] = ord("C") if region[50] == ord("A") else ord("A")
    tg = O.Target(target, A.ALPHABET_PROTEIN)
    from phraya_b200.batch import PackedReads
    packed = PackedReads([bytes(region)])
    rr, aln, cig, _ = tg.align_packed(packed, A.SENSITIVE, A.GAP_AFFINE, nthreads=1)
    assert rr[0]["has_result"] == 1 and rr[0]["reverse"] == 0
    off, var, cov, al = tg.variants_packed(packed, rr, aln, cig, A.SENSITIVE)
    assert len(var) >= 1 and set(var["strand"].tolist()) == {0}


def test_anchors_from_chains_reference_cases():
    # executor.rs tests anchors_from_chains_falls_back_to_origin_when_no_chains and
    # anchors_from_chains_uses_chain_target_start_and_respects_cap (:1170-1239)
    assert O.anchors([], A.FAST) == [0]
    chains = [100, 5000, 9000]  # target starts of chains scored 30, 25, 20 (chain order)
    assert O.anchors(chains, A.FAST) == [100]
    assert O.anchors(chains, A.BALANCED) == [100, 5000]
    assert O.anchors(chains, A.SENSITIVE) == [100, 5000, 9000]


def test_canonical_sketch_is_strand_symmetric():
    """Canonical minimizers with odd l = w + k - 1 (README.md:190): a sequence and its
    reverse complement select the same k-mers, at mirrored positions, with the same
    canonical values (the property the window orientation rule exists for)."""
    import random
    rng = random.Random(5)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    for n in (40, 150, 1000, 5000):
        s = bytes(rng.choice(b"ACGT") for _ in range(n))
        v, p = O.sketch(s)
        rv, rp = O.sketch(s.translate(comp)[::-1])
        fwd = sorted(zip(p.tolist(), v.tolist()))
        back = sorted((n - 21 - int(q), int(x)) for q, x in zip(rp, rv))
        assert fwd == back, n
        assert len(fwd) > (n - 30) * 2 // 13 if n > 100 else True


def test_sketch_values_are_2bit_kmers():
    """Values are the 2-bit k-mers (A=0, C=1, T=2, G=3, first character lowest); DNA
    takes the smaller of the k-mer and its reverse complement; protein characters go
    through the same 2-bit code."""
    s = b"ACGTTGCAACGGTACCATGAC" * 3
    v, p = O.sketch(s)
    code = {ord("A"): 0, ord("C"): 1, ord("T"): 2, ord("G"): 3}
    for val, pos in zip(v.tolist(), p.tolist()):
        km = s[pos:pos + 21]
        f = sum(code[c] << (2 * i) for i, c in enumerate(km))
        r = sum((code[c] ^ 2) << (2 * (20 - i)) for i, c in enumerate(km))
        assert val == min(f, r)
    prot = b"MKVLAGHWEERTYIPQSDNCF" * 2
    pv, pp = O.sketch(prot, 6, 5, A.ALPHABET_PROTEIN)
    for val, pos in zip(pv.tolist(), pp.tolist()):
        assert val == sum(((c >> 1) & 3) << (2 * i) for i, c in enumerate(prot[pos:pos + 6]))
