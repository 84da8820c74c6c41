"""GPU parity of the extension engines (WFA linear/affine, Myers fitting/global)
against the CPU oracle, through the C ABI. Bit-exact: status, CIGAR, edit distance
and all four coordinates must be identical."""
import numpy as np
import pytest

import known
import oracle as O
import refgen as R
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D

pytestmark = pytest.mark.gpu
ENGINES = [A.ENGINE_WFA_LINEAR, A.ENGINE_WFA_AFFINE, A.ENGINE_MYERS_FIT, A.ENGINE_MYERS_GLOBAL]
NAMES = {0: "wfa", 1: "affine", 2: "myers_fit", 3: "myers_global"}


@pytest.fixture(scope="module")
def eng():
    e = P.Engine(0)
    yield e
    e.close()


def gpu_align(eng):
    def f(engine, q, t, qseed, tseed):
        return eng.extend(engine, [(q, t, qseed, tseed)])[0]
    return f


def compare(eng, engine, pairs, costs=(2, 4, 1)):
    packed = pairs if isinstance(pairs, O.PackedPairs) else O.PackedPairs(pairs)
    ga, gc = eng.extend_packed(engine, packed, P.AffineCosts(*costs))
    oa, oc = O.extend_packed(engine, packed, costs)
    g = P.unpack(ga, gc)
    o = P.unpack(oa, oc)
    bad = [i for i in range(packed.n) if g[i] != o[i]]
    if bad:
        i = bad[0]
        q = bytes(packed.seq[packed.q_off[i]:packed.q_off[i] + packed.q_len[i]])
        t = bytes(packed.seq[packed.t_off[i]:packed.t_off[i] + packed.t_len[i]])
        raise AssertionError(f"{NAMES[engine]}: {len(bad)}/{packed.n} differ; first #{i}\n gpu={g[i]}\n "
                             f"ref={o[i]}\n q={q[:400]!r}\n t={t[:400]!r}")
    if engine == A.ENGINE_WFA_AFFINE:
        assert np.array_equal(ga["affine_score"], oa["affine_score"])
    return g


KA = known.load()


@pytest.mark.parametrize("case", KA["cases"], ids=[c["src"] for c in KA["cases"]])
def test_known_answer_gpu(eng, case):
    known.check_case(case, gpu_align(eng))


@pytest.mark.parametrize("case", KA["pairs_equal"], ids=[c["src"] for c in KA["pairs_equal"]])
def test_engines_agree_gpu(eng, case):
    known.check_pair(case, gpu_align(eng))


@pytest.mark.parametrize("engine", ENGINES, ids=[NAMES[e] for e in ENGINES])
def test_reference_sweeps_bit_exact(eng, engine):
    cases = (R.scalar_edit_sweep() + R.affine_fitting_cases() + R.affine_global_cases() +
             R.myers_wfa_fitting_sweep())
    compare(eng, engine, cases)


@pytest.mark.parametrize("engine", ENGINES, ids=[NAMES[e] for e in ENGINES])
def test_microbench_pairs_bit_exact(eng, engine):
    packed = D.extension_pairs(3000, 100, 300, 0.05, seed=11)
    compare(eng, engine, packed)
    if engine == A.ENGINE_WFA_AFFINE:
        compare(eng, engine, packed, costs=(4, 6, 2))


def test_myers_long_pairs_bit_exact(eng):
    packed = D.extension_pairs(300, 64, 2048, 0.05, seed=12, log_uniform=True)
    compare(eng, A.ENGINE_MYERS_GLOBAL, packed)
    compare(eng, A.ENGINE_MYERS_FIT, packed)


def test_fitting_windows_and_seeds(eng):
    # read vs 2x window (fitting branch), anchors at nonzero offsets
    rng = np.random.default_rng(5)
    pairs = []
    for i in range(600):
        t = bytes(rng.choice(list(b"ACGT"), 700).tolist())
        ql = int(rng.integers(50, 300))
        s = int(rng.integers(0, 200))
        q = bytearray(t[s:s + ql])
        for _ in range(int(rng.integers(0, 6))):
            q[int(rng.integers(0, len(q)))] = int(rng.choice(list(b"ACGT")))
        pairs.append((bytes(q), t, 0, s if i % 3 else max(0, s - 3)))
    for e in ENGINES:
        compare(eng, e, pairs)


def test_high_divergence_and_unrelated(eng):
    # large scores exercise the overflow redo passes
    rng = np.random.default_rng(6)
    pairs = []
    for _ in range(120):
        ql, tl = int(rng.integers(20, 400)), int(rng.integers(20, 800))
        pairs.append((bytes(rng.choice(list(b"ACGT"), ql).tolist()), bytes(rng.choice(list(b"ACGT"), tl).tolist())))
    for e in ENGINES:
        compare(eng, e, pairs)


def test_multi_stripe_myers(eng):
    packed = D.extension_pairs(12, 2100, 4200, 0.03, seed=13)
    compare(eng, A.ENGINE_MYERS_GLOBAL, packed)
    compare(eng, A.ENGINE_MYERS_FIT, packed)


def test_byte_path_non_acgt(eng):
    # lowercase, N and protein letters take the byte path; comparisons stay exact bytes
    rng = np.random.default_rng(7)
    pairs = []
    alph = list(b"ACDEFGHIKLMNPQRSTVWY")
    for i in range(300):
        L = int(rng.integers(5, 500))
        q = bytearray(rng.choice(alph if i % 2 else list(b"ACGTN"), L).tolist())
        t = bytearray(q)
        for _ in range(int(rng.integers(0, 20))):
            p = int(rng.integers(0, len(t)))
            t[p] = int(rng.choice(alph))
        if i % 5 == 0:
            t = t.lower()
        if i % 7 == 0:
            t = t + bytes(rng.choice(alph, 300).tolist())
        pairs.append((bytes(q), bytes(t)))
    for e in ENGINES:
        compare(eng, e, pairs)


def test_edges(eng):
    pairs = [(b"", b""), (b"", b"ACGT"), (b"ACG", b""), (b"A", b"A"), (b"A", b"C"), (b"ACGT", b"ACGT", 4, 4),
             (b"ACGT", b"ACGT", 5, 0), (b"ACGT", b"ACGT", 0, 5), (b"ACGTACGT", b"ACGT", 8, 0), (b"N", b"N"),
             (b"ACGT" * 40, b"")]
    for e in ENGINES:
        compare(eng, e, pairs)
        compare(eng, e, pairs, costs=(4, 6, 2))


def test_percall_matches_batched(eng):
    packed = D.extension_pairs(40, 100, 300, 0.05, seed=14)
    for e in ENGINES:
        a1, c1 = eng.extend_packed(e, packed)
        a2, c2 = eng.extend_packed(e, packed, percall=True)
        assert P.unpack(a1, c1) == P.unpack(a2, c2)


def long_linear_pairs():
    """Pairs long enough for the CTA-per-pair linear WFA kernel (qlen+tlen >= 4096)."""
    rng = np.random.default_rng(21)
    packed = D.extension_pairs(40, 2100, 12000, 0.08, seed=21)
    pairs = [(bytes(packed.seq[packed.q_off[i]:packed.q_off[i] + packed.q_len[i]]),
              bytes(packed.seq[packed.t_off[i]:packed.t_off[i] + packed.t_len[i]])) for i in range(packed.n)]
    for i in range(12):  # fitting branch: read inside a window more than 1.5x its length
        t = bytes(rng.choice(list(b"ACGT"), 7000).tolist())
        s = int(rng.integers(0, 3000))
        q = bytearray(t[s:s + 2600])
        for _ in range(int(rng.integers(0, 120))):
            q[int(rng.integers(0, len(q)))] = int(rng.choice(list(b"ACGT")))
        pairs.append((bytes(q), t, 0, s if i % 2 else 0))
    for L in (2500, 5000):  # unrelated: scores near half the length, widest frames
        pairs.append((bytes(rng.choice(list(b"ACGT"), L).tolist()), bytes(rng.choice(list(b"ACGT"), L + 100).tolist())))
    q = bytes(rng.choice(list(b"ACGT"), 6000).tolist())
    pairs.append((q, q))                                     # identical
    qb = bytearray(q)
    for p in rng.integers(0, 6000, 40):
        qb[int(p)] = ord("N")
    pairs.append((bytes(qb), q.lower()))                     # byte path: N and lowercase
    pairs.append((bytes(qb[:3000]), bytes(qb)))              # byte path, fitting
    return pairs


def test_long_linear_pairs_cta_kernel(eng):
    pairs = long_linear_pairs()
    assert eng.get_tune("wfa_big_min") > 0
    compare(eng, A.ENGINE_WFA_LINEAR, pairs)
    # small shared memory: frames of the widest pairs move to global memory mid-run
    with P.Engine(0) as e2:
        e2.set_tune("wfa_big_smem", 40 << 10)
        compare(e2, A.ENGINE_WFA_LINEAR, pairs)
        # CTA kernel off: the warp-per-pair kernel on the same pairs
        e2.set_tune("wfa_big_min", 0)
        compare(e2, A.ENGINE_WFA_LINEAR, pairs)


def long_affine_pairs():
    """Gap-affine pairs long enough for the CTA-per-pair affine kernel (qlen+tlen >= 4096):
    global and fitting branches, seed offsets, the byte path."""
    rng = np.random.default_rng(22)
    packed = D.extension_pairs(10, 2100, 4000, 0.06, seed=22)
    pairs = [(bytes(packed.seq[packed.q_off[i]:packed.q_off[i] + packed.q_len[i]]),
              bytes(packed.seq[packed.t_off[i]:packed.t_off[i] + packed.t_len[i]])) for i in range(packed.n)]
    for i in range(4):  # fitting branch: read inside a window more than 1.5x its length
        t = bytes(rng.choice(list(b"ACGT"), 6000).tolist())
        s = int(rng.integers(0, 2000))
        q = bytearray(t[s:s + 2200])
        for _ in range(int(rng.integers(0, 60))):
            q[int(rng.integers(0, len(q)))] = int(rng.choice(list(b"ACGT")))
        pairs.append((bytes(q), t, 0, s if i % 2 else 0))
    q = bytes(rng.choice(list(b"ACGT"), 3000).tolist())
    pairs.append((q, q))                                     # identical
    qb = bytearray(q)
    for p in rng.integers(0, 3000, 30):
        qb[int(p)] = ord("N")
    pairs.append((bytes(qb), q.lower()[:2900] + q[2900:]))   # byte path
    return pairs


@pytest.mark.parametrize("costs", [(2, 4, 1), (4, 6, 2)])
def test_long_affine_pairs_cta_kernel(costs):
    pairs = long_affine_pairs()
    with P.Engine(0) as e:
        e.set_timing(True)
        compare(e, A.ENGINE_WFA_AFFINE, pairs, costs)
        assert e.kernel_times().get("wfa_affine_big", (0, 0.0))[0] >= 1
        # fewer threads per CTA (more CTAs per SM): the same results
        for threads in (512, 256):
            e.set_tune("wfa_affine_big_threads", threads)
            compare(e, A.ENGINE_WFA_AFFINE, pairs, costs)
        e.set_tune("wfa_affine_big_threads", 1024)
        # CTA kernel off: the warp-group kernel on the same pairs
        e.set_tune("wfa_big_min", 0)
        compare(e, A.ENGINE_WFA_AFFINE, pairs, costs)


def test_tune_keys_validated(eng):
    with pytest.raises(P.EngineError):
        eng.set_tune("no_such_key", 1)
    with pytest.raises(P.EngineError):
        eng.set_tune("wfa_group_long", 3)
    with pytest.raises(P.EngineError):
        eng.set_tune("block_threads", 512)
    with pytest.raises(P.EngineError):
        eng.set_tune("wfa_affine_big_threads", 768)
    before = eng.get_tune("myers_band_base")
    eng.set_tune("myers_band_base", before)
    assert eng.get_tune("myers_band_base") == before


@pytest.mark.parametrize("engine", ENGINES, ids=[NAMES[e] for e in ENGINES])
def test_protein_pairs_bit_exact(eng, engine):
    """protein_wfa_myers_edit_distance_agree (executor.rs:2001-2027): protein bytes run the
    byte path of every engine, bit-exact with the oracle; WFA and Myers agree on ed."""
    pairs = R.protein_wfa_myers_cases()
    g = compare(eng, engine, pairs)
    if engine in (A.ENGINE_WFA_LINEAR, A.ENGINE_MYERS_FIT):
        other = compare(eng, A.ENGINE_MYERS_FIT if engine == A.ENGINE_WFA_LINEAR else A.ENGINE_WFA_LINEAR, pairs)
        assert [x[2] for x in g] == [x[2] for x in other]
