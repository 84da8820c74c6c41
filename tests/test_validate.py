"""The size-independent result checks (phraya_b200.validate) on the CPU: the oracle's
results of every engine satisfy them, and mistakes planted in copies of those results
are counted under the property they break."""
import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import datagen as D
from phraya_b200 import validate as V
from phraya_b200.batch import PackedPairs


@pytest.fixture(scope="module")
def sets():
    pk = D.extension_pairs(1500, 100, 300, 0.05, seed=15)
    pb = D.extension_pairs(300, 64, 2048, 0.05, seed=16, log_uniform=True)
    rng = np.random.default_rng(17)
    seeded = []
    for _ in range(200):
        q = bytes(rng.choice(list(b"ACGT"), int(rng.integers(50, 400))).tolist())
        t = bytes(rng.choice(list(b"ACGT"), 30).tolist()) + q + bytes(
            rng.choice(list(b"ACGT"), int(rng.integers(0, 300))).tolist())
        qs = int(rng.integers(0, 20))
        seeded.append((q, t, qs, qs + 30))
    return pk, pb, PackedPairs(seeded)


CASES = [(A.ENGINE_WFA_AFFINE, (4, 6, 2)), (A.ENGINE_WFA_AFFINE, (2, 4, 1)), (A.ENGINE_WFA_LINEAR, (2, 4, 1)),
         (A.ENGINE_MYERS_FIT, (2, 4, 1)), (A.ENGINE_MYERS_GLOBAL, (2, 4, 1))]


@pytest.mark.parametrize("engine,costs", CASES)
def test_oracle_results_pass(sets, engine, costs):
    pk, pb, seeded = sets
    batches = [pb] if engine == A.ENGINE_MYERS_GLOBAL else [pk, seeded]
    for p in batches:
        aln, cig = O.extend_packed(engine, p, costs)
        r = V.check_extensions(engine, aln, cig, p.q_len, costs, p.t_len)
        assert r["checked"] == int((aln["status"] == A.PHR_OK).sum()) > 0
        assert r["violations"] == 0, r


def test_planted_mistakes_are_counted(sets):
    pk = sets[0]
    costs = (4, 6, 2)
    aln, cig = O.extend_packed(A.ENGINE_WFA_AFFINE, pk, costs)

    def check(a, c):
        return V.check_extensions(A.ENGINE_WFA_AFFINE, a, c, pk.q_len, costs)

    # edit distance off by one in one record
    a = aln.copy()
    a["edit_distance"][3] += 1
    assert check(a, cig)["edit_distance"] == 1
    # a target span one base short
    a = aln.copy()
    a["target_end"][5] -= 1
    assert check(a, cig)["target_span"] == 1
    # an affine score that is not the CIGAR's cost
    a = aln.copy()
    a["affine_score"][7] += 2
    assert check(a, cig)["affine_score"] == 1
    # a run letter that is not M, X, I or D
    c = cig.copy()
    i = int(aln["cigar_off"][9] + aln["cigar_len"][9] - 1)
    c[i] = ord("Q")
    assert check(aln, c)["cigar_malformed"] == 1
    # a run count of zero
    c = cig.copy()
    j = int(aln["cigar_off"][11])
    c[j] = ord("0")
    r = check(aln, c)
    assert r["cigar_malformed"] >= 1 and r["violations"] >= 1
    # failed pairs are not checked
    a = aln.copy()
    a["status"][:10] = A.PHR_ALIGNMENT_FAILED
    assert check(a, cig)["checked"] == aln.size - 10


def test_read_alignments_pass_and_plants_are_counted():
    """align_read results of the oracle (short and long reads, every strategy) pass the
    read-level checks; a planted start, end or distance mistake is counted."""
    ref = D.random_reference(200_000, seed=5)
    reads, _, _ = D.reads_on_reference(ref, 400, 150, 0.02, seed=6)
    lreads, _, _ = D.reads_on_reference(
        ref, 20, error=0.05, seed=8, sub_frac=0.4, max_indel=3,
        length_sampler=lambda g, n: np.clip(np.exp(g.normal(np.log(3000), 0.5, n)), 1000, 8000).astype(np.int64))
    otg = O.Target(ref)
    for rd in (reads, lreads):
        for strat in (A.BALANCED, A.SENSITIVE, A.FAST):
            rr, aln, cig, _ = otg.align_packed(rd, strat, A.GAP_AFFINE)
            r = V.check_read_alignments(rr, aln, cig, rd.len, len(ref))
            assert r["checked"] > 0 and r["violations"] == 0, r
    rr, aln, cig, _ = otg.align_packed(reads, A.BALANCED, A.GAP_AFFINE)
    a = aln.copy()
    a["query_start"][0] += 1
    a["target_end"][1] = len(ref) + 5
    a["edit_distance"][2] += 1
    r = V.check_read_alignments(rr, a, cig, reads.len, len(ref))
    assert r["query_start_not_zero"] == 1 and r["target_beyond_end"] == 1 and r["edit_distance"] == 1
    assert r["violations"] >= 3


def test_texts_not_back_to_back(sets):
    """Checking a subset whose texts are not adjacent in the arena (every other pair
    failed) reads them one by one and finds the same (clean) results, and still catches a
    planted mistake."""
    pk = sets[0]
    aln, cig = O.extend_packed(A.ENGINE_WFA_LINEAR, pk, (2, 4, 1))
    a = aln.copy()
    a["status"][::2] = A.PHR_ALIGNMENT_FAILED
    r = V.check_extensions(A.ENGINE_WFA_LINEAR, a, cig, pk.q_len)
    assert r["checked"] == aln.size // 2 and r["violations"] == 0, r
    a["edit_distance"][1] += 3
    assert V.check_extensions(A.ENGINE_WFA_LINEAR, a, cig, pk.q_len)["edit_distance"] == 1
