"""Parity at the shapes of the long-read and contig workloads (long reads on a
repeat-rich reference; contigs with SNPs, small indels and an inversion; protein pairs at
30 % substitution): the device path against the CPU oracle, bit for bit, at sizes the
oracle finishes in seconds."""
import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200.batch import PackedReads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = P.Engine(0)
    yield e
    e.close()


def repeat_reference(n, n_rep, seed):
    """Random DNA with n_rep copies of 1-5 kb segments pasted elsewhere at 0.5 % divergence."""
    rng = np.random.default_rng(seed)
    ref = bytearray(D.random_reference(n, seed=seed))
    for _ in range(n_rep):
        L = int(rng.integers(1000, 5001))
        src, dst = int(rng.integers(0, n - L)), int(rng.integers(0, n - L))
        unit = bytearray(ref[src:src + L])
        for _ in range(max(1, L // 200)):
            unit[int(rng.integers(0, L))] = int(rng.choice(list(b"ACGT")))
        ref[dst:dst + L] = unit
    return bytes(ref)


def contigs(ref, n, seed, lens=(50_000, 200_000)):
    """Contigs of a copy of `ref` carrying 0.5 % SNPs, 0.02 % 1-20 bp indels and one
    10-50 kb inversion."""
    rng = np.random.default_rng(seed)
    cp = bytearray(ref)
    for p in rng.integers(0, len(cp), len(cp) // 200):
        cp[int(p)] = int(rng.choice([c for c in b"ACGT" if c != cp[int(p)]]))
    out, last = bytearray(), 0
    for p in sorted(rng.integers(0, len(cp), len(cp) // 5000).tolist()):
        out += cp[last:p]
        L = int(rng.integers(1, 21))
        if rng.random() < 0.5:
            out += bytes(rng.choice(list(b"ACGT"), L).tolist())
            last = p
        else:
            last = p + L
    out += cp[last:]
    L = int(rng.integers(10_000, 50_001))
    s = int(rng.integers(0, len(out) - L))
    out[s:s + L] = bytes(out[s:s + L])[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    res = []
    for _ in range(n):
        L = int(rng.integers(*lens))
        s = int(rng.integers(0, len(out) - L))
        res.append(bytes(out[s:s + L]))
    return res


def compare(eng, idx, otg, packed, strat, gap=A.GAP_AFFINE, variants=False):
    g = eng.align_packed(idx, packed, strat, gap)
    o = otg.align_packed(packed, strat, gap)
    gr, orr = P.unpack_reads(*g[:3]), O.unpack_read_results(packed.n, *o[:3])
    bad = [i for i in range(packed.n) if gr[i] != orr[i]]
    assert not bad, f"{len(bad)} reads differ; first {bad[0]}: gpu={gr[bad[0]]} ref={orr[bad[0]]}"
    assert tuple(g[3]) == tuple(o[3])
    if variants:
        rr, aln, cig, _, off, var, cov, al = eng.align_packed_variants(idx, packed, strat, gap)
        ooff, ovar, ocov, oal = otg.variants_packed(packed, o[0], o[1], o[2], strat)
        assert off.tobytes() == ooff.tobytes() and var.tobytes() == ovar.tobytes()
        assert cov.tobytes() == ocov.tobytes() and al.tobytes() == oal.tobytes()
        assert len(var) > 0
    return gr


def test_long_reads_on_repeat_reference(eng):
    ref = repeat_reference(2_000_000, 20, 81)
    packed, _, _ = D.reads_on_reference(
        ref, 24, error=0.05, seed=82, sub_frac=0.4, max_indel=3,
        length_sampler=lambda g, n: np.clip(np.exp(g.normal(np.log(8000), 0.5, n)), 1000, 20000).astype(np.int64))
    idx = eng.index(ref)
    otg = O.Target(ref)
    compare(eng, idx, otg, packed, A.FAST)
    g = compare(eng, idx, otg, packed, A.BALANCED, variants=True)
    assert all(r[1] for r in g)
    few = PackedReads([bytes(packed.seq[o:o + l]) for o, l in zip(packed.off[:3], packed.len[:3])])
    compare(eng, idx, otg, few, A.SENSITIVE)
    compare(eng, idx, otg, few, A.SENSITIVE, A.GAP_LINEAR)


def test_contigs_with_inversion(eng):
    ref = D.random_reference(2_000_000, seed=91)
    packed = PackedReads(contigs(ref, 4, 92))
    idx = eng.index(ref)
    otg = O.Target(ref)
    for strat in (A.FAST, A.BALANCED):
        g = compare(eng, idx, otg, packed, strat)
        assert all(r[1] for r in g)


def test_protein_pairs_30_percent():
    rng = np.random.default_rng(93)
    aa = list(b"ACDEFGHIKLMNPQRSTVWY")
    pairs = []
    for _ in range(200):
        q = bytearray(rng.choice(aa, int(rng.integers(200, 801))).tolist())
        t = bytearray(q)
        for p in np.flatnonzero(rng.random(len(t)) < 0.3):
            t[int(p)] = int(rng.choice([c for c in aa if c != t[int(p)]]))
        pairs.append((bytes(q), bytes(t)))
    packed = O.PackedPairs(pairs)
    with P.Engine(0) as eng:
        for engine, costs in ((A.ENGINE_WFA_LINEAR, (2, 4, 1)), (A.ENGINE_WFA_AFFINE, (2, 4, 1)),
                              (A.ENGINE_MYERS_FIT, (2, 4, 1)), (A.ENGINE_MYERS_GLOBAL, (2, 4, 1))):
            ga, gc = eng.extend_packed(engine, packed, P.AffineCosts(*costs))
            oa, oc = O.extend_packed(engine, packed, costs)
            assert P.unpack(ga, gc) == P.unpack(oa, oc), engine
