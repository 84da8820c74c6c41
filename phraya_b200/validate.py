"""Size-independent consistency checks of extension results.

For a batch of any size, every alignment with status PHR_OK must satisfy properties
that need no second implementation to check:

  - its CIGAR text is a run list "<count><op>..." with ops in M, X, I, D and counts >= 1
    written without leading zeros;
  - the runs consume exactly the reported spans: M + X + D (D = query-extra base) equals
    query_end - query_start, and M + X + I (I = target-extra base) equals
    target_end - target_start (the letters of phraya-align/src/wfa_simd.rs:1101-1105);
  - edit_distance equals X + I + D, the Levenshtein distance of the CIGAR
    (levenshtein_from_cigar, phraya-align/src/wfa_simd.rs:893-908);
  - the whole query suffix after its seed is aligned: query_end equals the query length;
  - global Myers (PHR_ENGINE_MYERS_GLOBAL) spans both sequences whole;
  - gap-affine WFA: affine_score equals mismatch x X + the sum over gap runs of
    gap_open + gap_extend x run length (a gap of length L costs O + L E,
    phraya-align/src/wfa_simd.rs:521-540).

Everything is vectorised with numpy, so millions of results check in seconds.
"""
import numpy as np

from . import _abi as A

_OPS = np.frombuffer(b"MXID", dtype=np.uint8)


def parse_runs(aln, cigar, idx):
    """Run lists of the alignments `idx` (indices into aln): -> (owner, count, op, bad)
    with one entry per run (owner = position in idx, op 0..3 for M, X, I, D) and bad[i]
    true when alignment idx[i]'s text is not a well-formed run list."""
    cig = np.asarray(cigar, dtype=np.uint8)
    off = aln["cigar_off"][idx].astype(np.int64)
    ln = aln["cigar_len"][idx].astype(np.int64)
    n = len(idx)
    bad = ln == 0
    total = int(ln.sum())
    if total == 0:
        e = np.zeros(0, dtype=np.int64)
        return e, e, e, bad
    starts = np.cumsum(ln) - ln  # of each text in the concatenation
    if (off[0] + total <= cig.size) and (n == 1 or np.array_equal(off[1:], off[:-1] + ln[:-1])):
        b = cig[off[0]:off[0] + total]  # the texts lie back to back in the arena: a view
    else:
        pos = np.arange(total, dtype=np.int64) - np.repeat(starts, ln) + np.repeat(off, ln)
        if pos.max() >= cig.size:
            raise ValueError("a CIGAR reaches past the text arena")
        b = cig[pos]
    is_digit = (b >= ord("0")) & (b <= ord("9"))
    op_code = np.full(b.shape, -1, dtype=np.int8)
    for c, ch in enumerate(_OPS):
        op_code[b == ch] = c
    is_op = op_code >= 0
    # every byte is a digit or an op, and every text ends with an op
    stray = np.flatnonzero(~(is_digit | is_op))
    if stray.size:
        bad[np.searchsorted(starts, stray, side="right") - 1] = True
    nz = ~bad
    bad[nz] |= ~is_op[(starts + ln - 1)[nz]]
    op_at = np.flatnonzero(is_op)
    owner = np.searchsorted(starts, op_at, side="right") - 1
    # digits of each run: the bytes between the previous op of the same text (or the text's
    # start) and this op
    prev_end = np.empty_like(op_at)
    prev_end[0] = 0
    prev_end[1:] = op_at[:-1] + 1
    first_of_text = np.ones(op_at.size, dtype=bool)
    first_of_text[1:] = owner[1:] != owner[:-1]
    prev_end[first_of_text] = starts[owner[first_of_text]]
    ndig = op_at - prev_end
    count = np.zeros(op_at.size, dtype=np.int64)
    scale = np.ones(op_at.size, dtype=np.int64)
    for d in range(1, 10):
        use = np.flatnonzero(ndig >= d)
        if use.size == 0:
            break
        count[use] += (b[op_at[use] - d].astype(np.int64) - ord("0")) * scale[use]
        scale[use] *= 10
    # counts are >= 1 and written without leading zeros, with 1 to 9 digits
    has = ndig >= 1
    lead_zero = np.zeros(op_at.size, dtype=bool)
    lead_zero[has] = b[prev_end[has]] == ord("0")
    wrong = (ndig < 1) | (ndig > 9) | (count < 1) | lead_zero
    if wrong.any():
        bad[owner[wrong]] = True
    return owner, count, op_code[op_at].astype(np.int64), bad


def check_extensions(engine, aln, cigar, q_len, costs=None, t_len=None):
    """Checks every PHR_OK result of one extension call (aln: ALN_DTYPE records, cigar:
    the text arena, q_len / t_len: the query / target lengths of the batch's pairs;
    t_len is needed only for the global engine's whole-target check). Returns a dict with
    the number of results checked and, per property, the number that violate it."""
    ok = np.flatnonzero(aln["status"] == A.PHR_OK)
    owner, count, op, bad = parse_runs(aln, cigar, ok)
    n = ok.size
    sums = np.zeros((n, 4), dtype=np.int64)
    np.add.at(sums, (owner, op), count)
    m, x, i, d = sums[:, 0], sums[:, 1], sums[:, 2], sums[:, 3]
    a = aln[ok]
    q_span = a["query_end"].astype(np.int64) - a["query_start"].astype(np.int64)
    t_span = a["target_end"].astype(np.int64) - a["target_start"].astype(np.int64)
    out = {
        "checked": int(n),
        "cigar_malformed": int(bad.sum()),
        "query_span": int(((m + x + d) != q_span).sum()),
        "target_span": int(((m + x + i) != t_span).sum()),
        "edit_distance": int(((x + i + d) != a["edit_distance"].astype(np.int64)).sum()),
        "query_not_whole": int((a["query_end"].astype(np.int64) != np.asarray(q_len, dtype=np.int64)[ok]).sum()),
    }
    if engine == A.ENGINE_MYERS_GLOBAL:
        whole = (a["query_start"] == 0) & (a["target_start"] == 0)
        if t_len is not None:
            whole &= a["target_end"].astype(np.int64) == np.asarray(t_len, dtype=np.int64)[ok]
        out["global_not_whole"] = int((~whole).sum())
    if engine == A.ENGINE_WFA_AFFINE and costs is not None:
        X, O, E = costs
        gap = (op == 2) | (op == 3)
        cost = np.zeros(n, dtype=np.int64)
        np.add.at(cost, owner[gap], O + E * count[gap])
        cost += X * x
        out["affine_score"] = int((cost != a["affine_score"].astype(np.int64)).sum())
    out["violations"] = int(sum(v for k, v in out.items() if k != "checked"))
    return out


def check_read_alignments(rr, aln, cigar, read_len, target_len):
    """The same checks for align_read results (rr: READ_RESULT_DTYPE per read, whose
    alignments are aln[aln_off .. aln_off + n_aln)): every alignment of a read spans the
    whole read (query_start 0, query_end its length, in the orientation it was aligned
    in) and ends inside the target; plus well-formed CIGARs, consumed spans and edit
    distance = X + I + D. The alignments mix engines, so the affine score is not checked."""
    n_aln = np.asarray(rr["n_aln"], dtype=np.int64)
    first = np.asarray(rr["aln_off"], dtype=np.int64)
    owner = np.repeat(np.arange(len(rr), dtype=np.int64), n_aln)
    within = np.arange(owner.size, dtype=np.int64) - np.repeat(np.cumsum(n_aln) - n_aln, n_aln)
    idx = np.repeat(first, n_aln) + within
    sub = aln[idx]
    out = check_extensions(-1, sub, cigar, np.asarray(read_len, dtype=np.int64)[owner])
    ok = sub["status"] == A.PHR_OK
    out["query_start_not_zero"] = int(((sub["query_start"] != 0) & ok).sum())
    out["target_beyond_end"] = int(((sub["target_end"].astype(np.int64) > int(target_len)) & ok).sum())
    out["violations"] = int(sum(v for k, v in out.items() if k not in ("checked", "violations")))
    return out
