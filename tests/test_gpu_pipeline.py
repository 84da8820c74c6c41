"""GPU parity of the read pipeline (sketch -> seed -> chain -> extend -> select)
against the CPU oracle's align_read restatement, through the C ABI."""
import numpy as np
import pytest

import oracle as O
import refgen as R
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D

pytestmark = pytest.mark.gpu
STRATS = [(A.FAST, A.GAP_AFFINE), (A.BALANCED, A.GAP_AFFINE), (A.SENSITIVE, A.GAP_AFFINE), (A.SENSITIVE, A.GAP_LINEAR)]


@pytest.fixture(scope="module")
def eng():
    e = P.Engine(0)
    yield e
    e.close()


def revcomp(s):
    return s[::-1].translate(bytes.maketrans(b"ACGTacgt", b"TGCAtgca"))


def test_sketch_parity(eng):
    rng = np.random.default_rng(1)
    seqs = [bytes(rng.choice(list(b"ACGT"), int(rng.integers(0, 3000))).tolist()) for _ in range(60)]
    seqs += [b"ACGTNNNNacgtACGT" * 20, b"A" * 500, b"", b"ACGT" * 5]
    got = eng.sketch(seqs)
    for s, (v, p) in zip(seqs, got):
        ov, op = O.sketch(s)
        assert np.array_equal(v, ov) and np.array_equal(p, op), len(s)
    prot = [bytes(rng.choice(list(b"ACDEFGHIKLMNPQRSTVWY"), 400).tolist()) for _ in range(10)]
    for s, (v, p) in zip(prot, eng.sketch(prot, 6, 5, A.ALPHABET_PROTEIN)):
        ov, op = O.sketch(s, 6, 5, A.ALPHABET_PROTEIN)
        assert np.array_equal(v, ov) and np.array_equal(p, op)


def test_seed_chain_parity(eng):
    ref = D.random_reference(200_000, seed=3)
    unit = ref[5000:7000]
    target = ref + unit + ref[:3000] + unit  # repeats for multi-chain cases
    idx = eng.index(target)
    tv, tp = O.sketch(target)
    cap = O.occurrence_cap(tv, tp)
    assert idx.info()["occurrence_cap"] == cap
    packed, _, _ = D.reads_on_reference(target, 300, 150, 0.02, seed=4)
    reads = [bytes(packed.seq[o:o + l]) for o, l in zip(packed.off, packed.len)]
    reads += [revcomp(r) for r in reads[:50]] + [unit[100:1100], R.diverse_dna(150, 9)]
    sks = [O.sketch(r) for r in reads]
    got = eng.seed_chain(idx, sks)
    for (v, p), (nseed, chains) in zip(sks, got):
        seeds = O.find_seeds(tv, tp, v, p, cap)
        assert nseed == len(seeds)
        exp = O.chain_seeds(seeds)
        assert chains == exp


def _seed_parity(eng, idx, tv, tp, reads):
    cap = O.occurrence_cap(tv, tp)
    assert idx.info()["occurrence_cap"] == cap
    sks = [O.sketch(r) for r in reads]
    for (v, p), (nseed, chains) in zip(sks, eng.seed_chain(idx, sks)):
        seeds = O.find_seeds(tv, tp, v, p, cap)
        assert nseed == len(seeds)
        assert chains == O.chain_seeds(seeds)


def test_index_build_on_device(eng):
    # build_minimizer_index + seed_occurrence_cap from the device's own sketch and from a
    # caller sketch; a repeated unit makes the median occurrence count (and so the cap)
    # exceed the floor of 256
    unit = D.random_reference(3000, seed=61)
    target = D.random_reference(500, seed=62) + unit * 120 + D.random_reference(300, seed=63)
    tv, tp = O.sketch(target)
    reads = [target[s:s + 150] for s in range(0, len(target) - 150, 9973)] + [unit[100:400], target[:400]]
    idx = eng.index(target)
    inf = idx.info()
    assert inf["n_minimizers"] == len(tv) and inf["n_distinct"] == len(np.unique(tv))
    assert inf["occurrence_cap"] > 256
    _seed_parity(eng, idx, tv, tp, reads)
    idx.close()
    # caller sketch: the device sketch's entries with a few positions moved, so the
    # position lists come from the caller's arrays, in the caller's order
    cv, cp = tv.copy(), tp.copy()
    cp[::7] = (cp[::7] + 3) % len(target)
    idx = eng.index(target, sketch=(cv, cp))
    assert idx.info()["n_distinct"] == len(np.unique(cv))
    _seed_parity(eng, idx, cv, cp, reads)
    idx.close()
    # empty sketch and a target shorter than k
    for t, sk in ((target[:5000], (np.zeros(0, np.uint64), np.zeros(0, np.uint32))), (b"ACGTACGT", None)):
        idx = eng.index(t, sketch=sk)
        inf = idx.info()
        assert inf["n_minimizers"] == 0 and inf["n_distinct"] == 0 and inf["occurrence_cap"] == 256
        assert eng.seed_chain(idx, [O.sketch(target[:150])])[0][0] == 0
        idx.close()


def compare_reads(eng, target, reads, strat, gap, stored=None, alphabet=A.ALPHABET_DNA):
    idx = eng.index(target, alphabet)
    otg = O.Target(target, alphabet)
    g, gst = eng.align_reads(idx, reads, strat, gap, stored=stored)
    o, ost = otg.align_reads(reads, strat, gap, stored=stored)
    bad = [i for i in range(len(reads)) if g[i] != o[i]]
    assert not bad, f"{len(bad)} reads differ; first {bad[0]}:\n gpu={g[bad[0]]}\n ref={o[bad[0]]}\n read={reads[bad[0]]!r}"
    assert gst == ost
    return g


@pytest.mark.parametrize("strat,gap", STRATS, ids=["fast", "balanced", "sensitive_affine", "sensitive_linear"])
def test_align_reads_reference_scenarios(eng, strat, gap):
    # chaining_correctness.rs:41-154 and executor.rs:1333-1438 scenarios
    t1 = R.diverse_dna(300, 1)
    r1 = bytearray(t1[50:200])
    r1[30] = ord("C") if r1[30] == ord("A") else ord("A")
    compare_reads(eng, t1, [bytes(r1)], strat, gap)
    t2 = R.diverse_dna(300, 2)
    r2 = bytearray(t2[50:200])
    del r2[60]
    compare_reads(eng, t2, [bytes(r2)], strat, gap)
    unit = R.diverse_dna(200, 3)
    t3 = unit + R.diverse_dna(500, 4) + unit + R.diverse_dna(500, 6)
    compare_reads(eng, t3, [unit[20:170]], strat, gap)
    compare_reads(eng, R.diverse_dna(300, 5), [R.diverse_dna(150, 999)], strat, gap)
    t7 = R.diverse_dna(300, 7)
    reg = bytearray(t7[100:200])
    reg[50] = ord("C") if reg[50] == ord("A") else ord("A")
    compare_reads(eng, t7, [revcomp(bytes(reg))], strat, gap)
    t8 = R.diverse_dna(300, 3)
    div = bytearray(t8[50:200])
    for i in range(67, 82):
        div[i] = ord("C") if div[i] == ord("A") else ord("A")
    compare_reads(eng, t8, [t8[50:150], bytes(div), R.diverse_dna(120, 987654)], strat, gap)


@pytest.mark.parametrize("strat,gap", STRATS, ids=["fast", "balanced", "sensitive_affine", "sensitive_linear"])
def test_align_reads_synthetic_case2(eng, strat, gap):
    ref = D.random_reference(300_000, seed=11)
    target = ref + ref[1000:4000]  # a repeat copy for multi-mapping
    packed, _, _ = D.reads_on_reference(target, 1500, 150, 0.01, seed=12)
    reads = [bytes(packed.seq[o:o + l]) for o, l in zip(packed.off, packed.len)]
    longp, _, _ = D.reads_on_reference(target, 40, 900, 0.03, seed=13)
    reads += [bytes(longp.seq[o:o + l]) for o, l in zip(longp.off, longp.len)]
    reads += [R.diverse_dna(150, 77), b"", b"ACGT", b"N" * 150]
    compare_reads(eng, target, reads, strat, gap)


def test_align_reads_stored_sketches(eng):
    target = D.random_reference(50_000, seed=21)
    packed, _, _ = D.reads_on_reference(target, 100, 150, 0.01, seed=22)
    reads = [bytes(packed.seq[o:o + l]) for o, l in zip(packed.off, packed.len)]
    stored = []
    for i, r in enumerate(reads):
        if i % 3 == 0:
            stored.append(None)
        elif i % 3 == 1:
            stored.append(O.sketch(r))
        else:
            stored.append((np.zeros(0, np.uint64), np.zeros(0, np.uint32)))
    compare_reads(eng, target, reads, A.BALANCED, A.GAP_AFFINE, stored=stored)


def test_align_reads_protein(eng):
    rng = np.random.default_rng(31)
    alph = list(b"ACDEFGHIKLMNPQRSTVWY")
    target = bytes(rng.choice(alph, 20000).tolist())
    reads = []
    for _ in range(60):
        s = int(rng.integers(0, 19000))
        r = bytearray(target[s:s + int(rng.integers(200, 800))])
        for _ in range(len(r) // 10):
            r[int(rng.integers(0, len(r)))] = int(rng.choice(alph))
        reads.append(bytes(r))
    reads.append(bytes(rng.choice(alph, 300).tolist()))
    for strat, gap in STRATS:
        compare_reads(eng, target, reads, strat, gap, alphabet=A.ALPHABET_PROTEIN)
