"""The benchmark-case generators: the restated read simulator reproduces the reference
simulator's output (digests in tests/golden/case2_digests.json, written by
tests/golden/make_case2_digests.py from scripts/benchmark/local/gen_synthetic.py), and
the long-read and contig generators have the stated shapes."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

from phraya_b200 import casegen as G

GOLD = os.path.join(os.path.dirname(__file__), "golden", "case2_digests.json")


def sha(s):
    return hashlib.sha256(s.encode()).hexdigest()


def golden():
    with open(GOLD) as fh:
        return json.load(fh)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_case2_short_matches_reference_simulator(k):
    g = golden()["sets"][k]
    p = g["params"]
    c = G.case2_short(**p)
    assert len(c.reads) == g["n_reads"]
    assert sha(c.genome.decode()) == g["genome_sha256"]
    assert sha("\n".join(r.decode() for r in c.reads)) == g["reads_sha256"]
    truth = [f"{s}\t{'-' if r else '+'}\t{n}\t" + ";".join(f"{o}:{op}:{ln}" for o, op, ln in ev)
             for s, r, n, ev in zip(c.starts, c.reverse, c.n_subs, c.indels)]
    assert sha("\n".join(truth)) == g["truth_sha256"]


def test_mutation_walk_protein_alphabet_matches_reference():
    for case in golden()["protein_mutations"]:
        rng = random.Random(case["seed"])
        frag = "".join(rng.choices(G.AMINO_ACIDS, k=case["length"]))
        mut, n_subs, ev = G.mutate_sites(frag, case["divergence"], case["indel_rate"], case["indel_max_len"], rng,
                                         alphabet=G.AMINO_ACIDS)
        assert sha(mut) == case["mutated_sha256"]
        assert n_subs == case["n_subs"]
        assert [list(e) for e in ev] == case["events"]


def test_case2_short_reads_come_from_the_genome():
    c = G.case2_short(genome_size=20_000, num_reads=200, read_len=150, divergence=0.0, indel_rate=0.0, seed=3)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    for r, s, rev in zip(c.reads, c.starts, c.reverse):
        frag = c.genome[s:s + 150]
        assert r == (frag.translate(comp)[::-1] if rev else frag)


def test_protein_pairs_shape():
    pairs = G.protein_pairs(200, seed=1)
    assert all(200 <= len(t) <= 800 and len(q) == len(t) for q, t in pairs)
    diff = sum(a != b for q, t in pairs for a, b in zip(q, t)) / sum(len(t) for _, t in pairs)
    assert 0.27 < diff < 0.33
    assert set(b"".join(q for q, _ in pairs)) <= set(G.AMINO_ACIDS.encode())


def test_long_read_and_contig_shapes():
    ref = G.repeat_reference(400_000, 5, seed=2)
    assert len(ref) == 400_000
    packed, starts, rev = G.long_reads(ref, 400, seed=3)
    lens = packed.len.astype(np.int64)
    assert lens.min() >= 900 and lens.max() <= 55_000
    assert 6000 < np.median(lens) < 10_000
    contigs = G.contig_set(ref, 12, seed=4, n_inversions=1)
    total = sum(len(c) for c in contigs)
    assert abs(total - len(ref)) < len(ref) * 0.01
    assert len(contigs) == 12 and G.n50([len(c) for c in contigs]) > total / 12
