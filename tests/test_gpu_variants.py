"""GPU parity of the variant-observation step (phr_align_reads_variants) and of the
index's tandem-repeat regions (phr_index_repeat_regions) against the CPU oracle, bit
for bit: every field of every observation, local coverage and allele list, the f64
confidence included."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import refgen as R
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200.batch import PackedReads

pytestmark = pytest.mark.gpu
STRATS = [(A.FAST, A.GAP_AFFINE), (A.BALANCED, A.GAP_AFFINE), (A.SENSITIVE, A.GAP_AFFINE), (A.SENSITIVE, A.GAP_LINEAR)]


@pytest.fixture(scope="module")
def eng():
    e = P.Engine(0)
    yield e
    e.close()


def revcomp(s):
    return s[::-1].translate(bytes.maketrans(b"ACGTacgt", b"TGCAtgca"))


def str_target(n, seed):
    """Random DNA with planted short tandem repeats, lowercase stretches and N runs."""
    rng = np.random.default_rng(seed)
    t = bytearray(D.random_reference(n, seed=seed))
    for _ in range(n // 400):
        p = int(rng.integers(0, n - 200))
        period = int(rng.integers(1, 6))
        unit = bytes(rng.choice(list(b"ACGT"), period).tolist())
        reps = int(rng.integers(2, 12))
        blob = (unit * reps)[: n - p]
        t[p:p + len(blob)] = blob
    for _ in range(n // 5000):
        p = int(rng.integers(0, n - 100))
        t[p:p + 60] = bytes(t[p:p + 60]).lower()
    for _ in range(n // 20000):
        p = int(rng.integers(0, n - 300))
        w = int(rng.integers(10, 300))
        t[p:p + w] = b"N" * w
    return bytes(t)


def sim_reads(target, n, length, err, seed):
    """Reads copied from `target` with substitutions, insertions and deletions at rate `err`."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        p = int(rng.integers(0, len(target) - length))
        src = target[p:p + length + 20]
        r = bytearray()
        i = 0
        while len(r) < length and i < len(src):
            u = rng.random()
            if u < err * 0.6:
                r.append(int(rng.choice(list(b"ACGT"))))
                i += 1
            elif u < err * 0.8:
                r += bytes(rng.choice(list(b"ACGT"), int(rng.integers(1, 5))).tolist())
            elif u < err:
                i += int(rng.integers(1, 5))
            else:
                r.append(src[i])
                i += 1
        out.append(bytes(r))
    return out


def test_repeat_regions_parity(eng):
    seqs = [s for s, _ in [
        (b"ATATATATAT", 0), (b"CAGCAGCAGCAG", 0), (b"GATAGATAGATA", 0), (b"GCGCGCGC", 0), (b"AAAAAAAAA", 0),
        (b"ATGCATGATCGATCG", 0), (b"AtAtAtAtAt", 0), (b"ACACACACACGT", 0), (b"AAAAAAAAAAAAAA", 0)]]
    seqs += [str_target(200_000, 1), str_target(50_000, 2), b"N" * 5000 + D.random_reference(3000, seed=3),
             b"ACGT" * 2000, b"A" * 7]
    for s in seqs:
        idx = eng.index(s)
        assert idx.repeat_regions() == O.tandem_repeats(s), len(s)
        idx.close()


def test_repeat_regions_protein_index(eng):
    rng = np.random.default_rng(5)
    t = bytearray(rng.choice(list(b"ACDEFGHIKLMNPQRSTVWY"), 20000).tolist())
    t[100:124] = b"QQQQ" * 6
    t[500:518] = b"KRE" * 6
    idx = eng.index(bytes(t), A.ALPHABET_PROTEIN)
    assert idx.repeat_regions() == O.tandem_repeats(bytes(t))


def compare_variants(eng, target, reads, strat, gap, radius=0, hotspots=(), stored=None, alphabet=A.ALPHABET_DNA):
    idx = eng.index(target, alphabet)
    otg = O.Target(target, alphabet)
    packed = PackedReads(reads, stored)
    rr, aln, cig, st, off, var, cov, al = eng.align_packed_variants(idx, packed, strat, gap, radius, hotspots)
    # the alignments are phr_align_reads' own
    rr2, aln2, cig2, st2 = eng.align_packed(idx, packed, strat, gap)
    assert rr.tobytes() == rr2.tobytes() and aln.tobytes() == aln2.tobytes() and cig.tobytes() == cig2.tobytes()
    assert st == st2
    # the oracle's observations of the oracle's own alignments
    orr, oaln, ocig, ost = otg.align_packed(packed, strat, gap)
    assert P.unpack_reads(rr, aln, cig) == O.unpack_read_results(packed.n, orr, oaln, ocig)
    ooff, ovar, ocov, oal = otg.variants_packed(packed, orr, oaln, ocig, strat, radius, hotspots)
    assert np.array_equal(off, ooff)
    bad = [i for i in range(len(var)) if var[i].tobytes() != ovar[i].tobytes()] if len(var) == len(ovar) else [-1]
    assert not bad, f"{len(bad)} observations differ; first {bad[0]}: gpu={var[bad[0]]} ref={ovar[bad[0]]}"
    assert np.array_equal(cov, ocov)
    assert al.tobytes() == oal.tobytes()
    return off, var, cov, al


@pytest.mark.parametrize("strat,gap", STRATS, ids=["fast", "balanced", "sensitive_affine", "sensitive_linear"])
def test_variants_parity_synthetic(eng, strat, gap):
    ref = str_target(120_000, 11)
    target = ref + ref[1000:4000] + ref[9000:9800]  # repeat copies: multi-mapped reads, alternatives
    reads = sim_reads(target, 700, 150, 0.03, 12)
    reads += [revcomp(r) for r in reads[:200]]
    reads += sim_reads(target, 20, 900, 0.04, 13)
    reads += [R.diverse_dna(150, 77), b"", b"ACGT", b"N" * 150, ref[2000:2150].lower()]
    hot = [(s, s + int(w)) for s, w in zip(range(500, len(target) - 400, 2500), [3, 40, 200, 1] * 200)]
    off, var, cov, al = compare_variants(eng, target, reads, strat, gap, hotspots=hot)
    assert len(var) > 500
    types = set(var["variant_type"].tolist())
    assert types == {0, 1, 2}
    assert set(var["strand"].tolist()) == {0, 1}
    assert (var["kmer_uniqueness"] == 0.0).any() and (var["in_tandem_repeat"] == 1).any()


def test_variants_parity_radius_and_scenarios(eng):
    # executor.rs / local_coverage_tests.rs scenarios with explicit and default radii
    t1 = R.diverse_dna(300, 1)
    r1 = bytearray(t1[50:200])
    r1[30] = ord("C") if r1[30] == ord("A") else ord("A")
    t2 = R.diverse_dna(300, 2)
    r2 = bytearray(t2[50:200])
    del r2[60]
    for radius in (0, 1, 7, 400):
        compare_variants(eng, t1, [bytes(r1), revcomp(bytes(r1))], A.BALANCED, A.GAP_AFFINE, radius=radius)
        compare_variants(eng, t2, [bytes(r2)], A.SENSITIVE, A.GAP_AFFINE, radius=radius)
    base = b"ACGT" * 45
    t = bytearray(base)
    t[75] = ord("A")
    compare_variants(eng, bytes(t), [base], A.BALANCED, A.GAP_AFFINE)
    t = bytearray(b"A" * 150)
    t[149] = ord("T")
    compare_variants(eng, bytes(t), [b"A" * 150], A.BALANCED, A.GAP_AFFINE)


def test_variants_parity_protein(eng):
    rng = np.random.default_rng(71)
    alph = list(b"ACDEFGHIKLMNPQRSTVWY")
    target = bytearray(rng.choice(alph, 30000).tolist())
    target[5000:5024] = b"QQQQ" * 6  # a tandem repeat on the protein index too
    target = bytes(target)
    reads = []
    for _ in range(150):
        p = int(rng.integers(0, len(target) - 400))
        r = bytearray(target[p:p + int(rng.integers(150, 400))])
        for _ in range(int(rng.integers(0, 12))):
            j = int(rng.integers(0, len(r)))
            u = rng.random()
            if u < 0.6:
                r[j] = int(rng.choice(alph))
            elif u < 0.8:
                r[j:j] = bytes(rng.choice(alph, int(rng.integers(1, 4))).tolist())
            else:
                del r[j:j + int(rng.integers(1, 4))]
        reads.append(bytes(r))
    for strat, gap in ((A.BALANCED, A.GAP_AFFINE), (A.SENSITIVE, A.GAP_AFFINE)):
        off, var, cov, al = compare_variants(eng, target, reads, strat, gap, hotspots=[(4000, 6000)],
                                             alphabet=A.ALPHABET_PROTEIN)
        assert len(var) > 100 and set(var["strand"].tolist()) == {0}


def test_variants_capacity_reports_needed_sizes(eng):
    target = D.random_reference(30_000, seed=41)
    packed, _, _ = D.reads_on_reference(target, 50, 150, 0.03, seed=42)
    idx = eng.index(target)
    n = packed.n
    rr = np.zeros(n, dtype=P.READ_RESULT_DTYPE)
    aln = np.empty(4 * n + 16, dtype=P.ALN_DTYPE)
    cig = np.empty(4 * (6 * int(packed.len.sum()) + 16 * n), dtype=np.uint8)
    off = np.zeros(n + 1, dtype=np.uint64)
    var = np.empty(1, dtype=P.VARIANT_DTYPE)
    cov = np.empty(1, dtype=np.uint32)
    al = np.empty(1, dtype=P.ALLELE_DTYPE)
    va = A.VariantArena(off.ctypes.data, var.ctypes.data, 1, 0, cov.ctypes.data, 1, 0, al.ctypes.data, 1, 0)
    arena = A.ReadResultArena(rr.ctypes.data, aln.ctypes.data, len(aln), 0, cig.ctypes.data, len(cig), 0)
    cfg = A.AlignConfig(A.BALANCED, A.GAP_AFFINE)
    b = packed.batch()
    st = eng._lib.phr_align_reads_variants(eng.handle, idx.handle, C.byref(b), C.byref(cfg), C.byref(arena), None,
                                           C.byref(va), None)
    assert st == A.PHR_ERR_CAPACITY
    _, _, _, _, off2, var2, cov2, al2 = eng.align_packed_variants(idx, packed, A.BALANCED, A.GAP_AFFINE)
    assert (va.variant_used, va.coverage_used, va.allele_used) == (len(var2), len(cov2), len(al2))


@pytest.mark.parametrize("mode", [A.COVERAGE_QUANTIZED, A.COVERAGE_DEPTH], ids=["quantized", "depth"])
def test_coverage_track_parity(eng, mode):
    ref = str_target(100_000, 51)
    target = ref + ref[2000:5000]
    idx = eng.index(target)
    track = eng.coverage_track(idx, mode)
    exp = np.zeros(len(target), dtype=np.uint32)
    for seed in (52, 53, 54):  # three batches merged into one resident track
        packed = PackedReads(sim_reads(target, 400, 150, 0.02, seed) + sim_reads(target, 10, 2000, 0.03, seed))
        rr, aln, cig, _ = eng.align_packed(idx, packed, A.SENSITIVE, A.GAP_AFFINE)
        track.add(aln)
        O.coverage_merge(aln, len(target), mode == A.COVERAGE_DEPTH, exp)
    got = track.read()
    assert np.array_equal(got, exp)
    assert got.any() == (mode == A.COVERAGE_DEPTH)
    track.close()


def test_protein_alignment_never_reverse(eng):
    # protein_alignment_never_attempts_reverse_strand (executor.rs:1965-1995)
    target = R.diverse_protein(300, 11)
    region = bytearray(target[100:200])
    region[50] = ord("C") if region[50] == ord("A") else ord("A")
    off, var, cov, al = compare_variants(eng, target, [bytes(region)], A.SENSITIVE, A.GAP_AFFINE,
                                         alphabet=A.ALPHABET_PROTEIN)
    assert len(var) >= 1 and set(var["strand"].tolist()) == {0}
