"""Seeded workloads of the reference's benchmark cases.

* `case2_short` restates the reference's read simulator
  (scripts/benchmark/local/gen_synthetic.py:33-193): one `random.Random(seed)` stream
  draws the i.i.d. ACGT genome, then per read a start, a strand and the per-site
  mutation events, so a given parameter set yields the same genome and reads as that
  script. `mutate_sites` is its per-site event walk (gen_synthetic.py:46-105), shared
  with `protein_pairs` as the protein generator shares it
  (scripts/benchmark/local/gen_synthetic_protein.py:28-29,82-84).
* `repeat_reference`, `long_reads`: the long-read case (a 5 Mbp genome with 20 pasted
  1-5 kb repeat copies at 0.5 % divergence; reads lognormal around 8 kb at 5 % error,
  60 % indels and 40 % substitutions, both strands). The reference has no generator for
  this case; numpy stands in.
* `contig_set`: the contig-to-reference case (a copy of the genome carrying 0.5 % SNPs,
  0.02 % 1-20 bp indels and inversions of 10-50 kb, cut into contigs of lognormal length
  that tile the copy once).
* `protein_pairs`: query/target protein pairs over the 20 canonical residues at a
  substitution divergence.
"""
import random

import numpy as np

from . import datagen as D
from .batch import PackedReads

DNA = "ACGT"
AMINO_ACIDS = "ACDEFGHIKLMNPQRSTVWY"
_COMP = str.maketrans("ACGT", "TGCA")


def mutate_sites(frag, divergence, indel_rate, indel_max_len, rng, alphabet=DNA):
    """Walks `frag` left to right with at most one event per original site: an indel
    (tested first, only when indel_rate > 0, so an indel-free run draws nothing for it)
    or a substitution by another symbol of `alphabet`. An insertion puts `length` random
    symbols before the site and visits the site again; a deletion skips up to `length`
    sites. Returns (mutated, n_subs, [(site, "I"|"D", length), ...])
    (gen_synthetic.py:46-105)."""
    out = []
    events = []
    n_subs = 0
    n = len(frag)
    i = 0
    rand, randint, choice, choices = rng.random, rng.randint, rng.choice, rng.choices
    while i < n:
        here = frag[i]
        if indel_rate > 0.0 and rand() < indel_rate:
            length = randint(1, indel_max_len)
            if rand() < 0.5:
                out.append("".join(choices(alphabet, k=length)))
                events.append((i, "I", length))
            else:
                length = min(length, n - i)
                events.append((i, "D", length))
                i += length
            continue
        if divergence > 0.0 and rand() < divergence:
            alt = choice(alphabet)
            while alt == here:
                alt = choice(alphabet)
            out.append(alt)
            n_subs += 1
        else:
            out.append(here)
        i += 1
    return "".join(out), n_subs, events


class Case2Reads:
    """Genome + single-end reads of the read-vs-reference case (Case 2)."""

    def __init__(self, genome, reads, starts, reverse, n_subs, indels):
        self.genome = genome          # bytes
        self.reads = reads            # list of bytes
        self.starts = starts          # genome start of each read's source fragment
        self.reverse = reverse        # True: the read is the reverse complement
        self.n_subs = n_subs
        self.indels = indels          # per read [(site, "I"|"D", length)]


def case2_short(genome_size=1_000_000, num_reads=20_000, read_len=150, divergence=0.01, indel_rate=0.0,
                indel_max_len=5, seed=1):
    """The reference simulator's genome and reads for these parameters
    (gen_synthetic.py:108-193; its defaults are genome 2,000,000, indel length 5, seed 1)."""
    if read_len > genome_size:
        raise ValueError(f"read_len {read_len} exceeds genome size {genome_size}")
    rng = random.Random(seed)
    genome = "".join(rng.choices(DNA, k=genome_size))
    last = genome_size - read_len
    reads, starts, rev, subs, indels = [], [], [], [], []
    for _ in range(num_reads):
        s = rng.randint(0, last)
        frag = genome[s:s + read_len]
        minus = rng.random() < 0.5
        if minus:
            frag = frag.translate(_COMP)[::-1]
        mut, ns, ev = mutate_sites(frag, divergence, indel_rate, indel_max_len, rng)
        reads.append(mut.encode())
        starts.append(s)
        rev.append(minus)
        subs.append(ns)
        indels.append(ev)
    return Case2Reads(genome.encode(), reads, starts, rev, subs, indels)


def protein_pairs(n=5000, lo=200, hi=800, divergence=0.30, seed=0):
    """n (query, target) pairs: the target i.i.d. over the 20 residues with length
    uniform in [lo, hi], the query the target with per-site substitutions at
    `divergence` (no indels)."""
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        t = "".join(rng.choices(AMINO_ACIDS, k=rng.randint(lo, hi)))
        q, _, _ = mutate_sites(t, divergence, 0.0, 1, rng, alphabet=AMINO_ACIDS)
        out.append((q.encode(), t.encode()))
    return out


def repeat_reference(n, n_rep, seed, rep_len=(1000, 5000), divergence=0.005):
    """i.i.d. ACGT genome of n bases with n_rep copies of rep_len-long segments pasted
    elsewhere, each copy carrying substitutions at `divergence`."""
    rng = np.random.default_rng(seed)
    ref = bytearray(D.random_reference(n, seed=seed))
    for _ in range(n_rep):
        L = int(rng.integers(rep_len[0], rep_len[1] + 1))
        src, dst = int(rng.integers(0, n - L)), int(rng.integers(0, n - L))
        unit = bytearray(ref[src:src + L])
        for _ in range(max(1, int(round(L * divergence)))):
            unit[int(rng.integers(0, L))] = int(rng.choice(list(b"ACGT")))
        ref[dst:dst + L] = unit
    return bytes(ref)


def lognormal_lengths(median, sigma, lo, hi):
    """Length sampler for datagen.reads_on_reference: lognormal, clipped to [lo, hi]."""
    return lambda g, n: np.clip(np.exp(g.normal(np.log(median), sigma, n)), lo, hi).astype(np.int64)


def _sorted_unique(a):
    a = np.sort(a)
    if a.size:
        a = a[np.concatenate(([True], a[1:] != a[:-1]))]
    return a


def _ranges(starts, lens):
    """Concatenation of the integer ranges [starts[i], starts[i] + lens[i])."""
    total = int(lens.sum())
    if total == 0:
        return np.zeros(0, dtype=np.int64)
    first = np.zeros(lens.size, dtype=np.int64)
    np.cumsum(lens[:-1], out=first[1:])
    return np.repeat(starts - first, lens) + np.arange(total, dtype=np.int64)


def mutate_sparse(rng, codes, seg_start, seg_len, rate, sub_frac, max_indel):
    """Mutates the concatenated segments of `codes` (values 0..3) with events at
    `rate` per base: a fraction sub_frac substitutions, the rest insertions and
    deletions in equal parts, of length uniform in [1, max_indel] (a deletion stops at
    its segment's end, an insertion goes before its site). Only the event sites are
    drawn and indexed, so the work beyond one copy of the sequence is proportional to
    the events. Returns (mutated codes, segment lengths)."""
    N = int(codes.size)
    seg_start = np.asarray(seg_start, dtype=np.int64)
    seg_len = np.asarray(seg_len, dtype=np.int64)
    seg_end = seg_start + seg_len
    pos = _sorted_unique(rng.integers(0, N, rng.binomial(N, rate))) if N else np.zeros(0, np.int64)
    kind = rng.random(pos.size)
    klen = rng.integers(1, max_indel + 1, pos.size)
    seg = np.searchsorted(seg_end, pos, side="right")
    half = sub_frac + (1.0 - sub_frac) / 2.0
    is_sub, is_ins, is_del = kind < sub_frac, (kind >= sub_frac) & (kind < half), kind >= half
    dl = np.minimum(pos + klen, seg_end[seg]) - pos
    gone = _sorted_unique(_ranges(pos[is_del], dl[is_del]))        # deleted sites, sorted
    keep = np.ones(N, dtype=bool)
    keep[gone] = False
    out = codes.astype(np.uint8, copy=True)
    sp = pos[is_sub & keep[pos]]
    out[sp] = (out[sp] + rng.integers(1, 4, sp.size).astype(np.uint8)) % 4
    ins_ok = is_ins & keep[pos]
    ip, il = pos[ins_ok], klen[ins_ok]
    kept_before = ip - np.searchsorted(gone, ip)                     # kept sites before each insertion site
    out = out[keep]
    ins = rng.integers(0, 4, int(il.sum())).astype(np.uint8)
    out = np.insert(out, np.repeat(kept_before, il), ins)
    dels = np.searchsorted(gone, seg_end) - np.searchsorted(gone, seg_start)
    ins_per = np.bincount(seg[ins_ok], weights=il, minlength=seg_start.size).astype(np.int64)
    return out, seg_len - dels + ins_per


def reads_from_genome(ref, lengths, rng, error, sub_frac, max_indel):
    """Reads of the given lengths at uniform starts on both strands of `ref`, mutated
    by mutate_sparse. Returns (PackedReads, starts, reverse)."""
    g = np.frombuffer(ref, dtype=np.uint8)
    codes = np.searchsorted(D.BASES, g).astype(np.uint8)
    lens = np.minimum(np.asarray(lengths, dtype=np.int64), g.size)
    n = lens.size
    starts = rng.integers(0, g.size - lens + 1)
    rev = rng.random(n) < 0.5
    seg_start = np.zeros(n, dtype=np.int64)
    np.cumsum(lens[:-1], out=seg_start[1:])
    src = np.concatenate([codes[s:s + L] for s, L in zip(starts.tolist(), lens.tolist())]) if n else codes[:0]
    mut, mlen = mutate_sparse(rng, src, seg_start, lens, error, sub_frac, max_indel)
    del src
    arena = D.BASES[mut]
    off = np.zeros(n, dtype=np.int64)
    np.cumsum(mlen[:-1], out=off[1:])
    comp = D.COMP
    for i in np.flatnonzero(rev).tolist():
        o, L = int(off[i]), int(mlen[i])
        arena[o:o + L] = comp[arena[o:o + L][::-1]]
    return PackedReads.from_arrays(arena, off.astype(np.uint64), mlen.astype(np.uint32)), starts, rev


def long_reads(ref, n, seed, median=8000, sigma=0.5, lo=1000, hi=50_000, error=0.05):
    """Long reads on both strands: lognormal lengths (median, sigma) clipped to [lo, hi],
    `error` per base with 40 % substitutions and 60 % indels of 1-3 bp.
    Returns (PackedReads, starts, reverse)."""
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(median, sigma, lo, hi)(rng, n)
    return reads_from_genome(ref, lens, rng, error, 0.4, 3)


def contig_set(ref, n_contigs, seed, n_inversions=3, inv_len=(10_000, 50_000), snp=0.005, indel=0.0002,
               indel_len=(1, 20), sigma=1.33):
    """Contigs of a copy of `ref`: SNPs at rate `snp`, indels of indel_len at rate
    `indel` per base, `n_inversions` reverse-complemented segments, then cut into
    n_contigs consecutive pieces of lognormal length (sigma 1.33 puts N50 near 2.4x the
    mean length, i.e. about 200 kb for 60 contigs over 5 Mbp). Returns a list of bytes."""
    rng = np.random.default_rng(seed)
    cp = np.frombuffer(ref, dtype=np.uint8).copy()
    codes = np.searchsorted(D.BASES, cp)
    sites = np.flatnonzero(rng.random(cp.size) < snp)
    cp[sites] = D.BASES[(codes[sites] + rng.integers(1, 4, sites.size)) % 4]
    out, last = [], 0
    for p in np.sort(rng.choice(cp.size, int(round(cp.size * indel)), replace=False)).tolist():
        if p < last:
            continue
        out.append(cp[last:p].tobytes())
        L = int(rng.integers(indel_len[0], indel_len[1] + 1))
        if rng.random() < 0.5:
            out.append(D.BASES[rng.integers(0, 4, L)].tobytes())
            last = p
        else:
            last = p + L
    out.append(cp[last:].tobytes())
    seq = bytearray(b"".join(out))
    for _ in range(n_inversions):
        L = int(rng.integers(inv_len[0], inv_len[1] + 1))
        s = int(rng.integers(0, len(seq) - L))
        seq[s:s + L] = bytes(seq[s:s + L])[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    w = np.exp(rng.normal(0.0, sigma, n_contigs))
    cuts = np.round(np.cumsum(w) / w.sum() * len(seq)).astype(np.int64)
    starts = np.concatenate([[0], cuts[:-1]])
    return [bytes(seq[a:b]) for a, b in zip(starts.tolist(), cuts.tolist()) if b > a]


def n50(lengths):
    """Length L such that contigs of length >= L hold half of the total."""
    ls = sorted(lengths, reverse=True)
    half, acc = sum(ls) / 2.0, 0
    for x in ls:
        acc += x
        if acc >= half:
            return x
    return 0
