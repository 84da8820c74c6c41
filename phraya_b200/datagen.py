"""Seeded synthetic workloads (numpy, vectorised).

The reference publishes no dataset for this path; these generators produce the shapes
and value distributions of the benchmark configurations instead:

* `extension_pairs` -- batched extension microbench pairs: query lengths uniform (or
  log-uniform) in [lo, hi], i.i.d. ACGT; each target is its query mutated at a per-pair
  divergence uniform in [0, max_div], events split 70 % substitutions / 30 % indels
  (insertions and deletions equally likely) of length uniform in [1, max_indel].
* `reads_on_reference` -- reads sampled at uniform positions on both strands of an
  i.i.d. reference, mutated like the pairs (the read-alignment pipeline workload).

All sequences are ASCII bytes in one arena with structure-of-arrays offsets, the layout
of phr_pair_batch / phr_read_batch.
"""
import ctypes

import numpy as np

from .batch import PackedPairs, PackedReads

# Keep freed large numpy buffers in the heap (no munmap) so repeated generation reuses
# already-mapped pages instead of faulting in fresh ones for every temporary.
try:
    _libc = ctypes.CDLL("libc.so.6")
    _libc.mallopt(-3, 1 << 30)  # M_MMAP_THRESHOLD
    _libc.mallopt(-1, 1 << 31)  # M_TRIM_THRESHOLD
except OSError:
    pass

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
COMP = np.zeros(256, dtype=np.uint8)
COMP[:] = np.arange(256, dtype=np.uint8)
for a, b in zip(b"ACGTacgt", b"TGCAtgca"):
    COMP[a] = b


def _mutate(rng, src, seg_start, seg_len, div, sub_frac=0.7, max_indel=5):
    """Mutates the concatenated segments of `src` (codes 0..3); returns (dst, dst_len)."""
    n = src.size
    pair_of = np.repeat(np.arange(seg_len.size), seg_len)
    d = div[pair_of]
    ev = rng.random(n) < d
    kind = rng.random(n)
    is_sub = ev & (kind < sub_frac)
    is_ins = ev & (kind >= sub_frac) & (kind < sub_frac + (1 - sub_frac) / 2)
    is_del = ev & (kind >= sub_frac + (1 - sub_frac) / 2)
    klen = rng.integers(1, max_indel + 1, n)
    pos = np.arange(n, dtype=np.int64)
    seg_end = (seg_start + seg_len)[pair_of]
    del_end = np.where(is_del, np.minimum(pos + klen, seg_end), 0)
    # a position is deleted when a deletion started at or before it (same segment) reaches past it
    run = np.maximum.accumulate(del_end)
    covered = run > pos
    keep = ~covered
    ins_len = np.where(is_ins & keep, klen, 0)
    per = keep.astype(np.int64) + ins_len
    out_off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(per, out=out_off[1:])
    total = int(out_off[-1])
    dst = rng.integers(0, 4, total).astype(np.uint8)  # inserted bases stay random
    kept_vals = src.copy()
    shift = rng.integers(1, 4, n).astype(np.uint8)
    kept_vals = np.where(is_sub, (kept_vals + shift) % 4, kept_vals).astype(np.uint8)
    kp = out_off[:-1][keep]
    dst[kp] = kept_vals[keep]
    seg_out = np.add.reduceat(per, seg_start) if n else np.zeros(0, np.int64)
    seg_out = np.where(seg_len > 0, seg_out, 0)
    return dst, seg_out.astype(np.int64)


def extension_pairs(n, lo=100, hi=300, max_div=0.05, seed=0, log_uniform=False, max_indel=5):
    """Query/target pairs for the batched extension microbench; returns PackedPairs."""
    rng = np.random.default_rng(seed)
    if log_uniform:
        qlen = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)
    else:
        qlen = rng.integers(lo, hi + 1, n)
    qlen = np.clip(qlen, lo, hi)
    div = rng.uniform(0.0, max_div, n)
    q_start = np.zeros(n, dtype=np.int64)
    np.cumsum(qlen[:-1], out=q_start[1:])
    q = rng.integers(0, 4, int(qlen.sum())).astype(np.uint8)
    t, tlen = _mutate(rng, q, q_start, qlen, div, max_indel=max_indel)
    # interleave q_i, t_i in one ASCII arena
    t_start = np.zeros(n, dtype=np.int64)
    np.cumsum(tlen[:-1], out=t_start[1:])
    arena = np.empty(q.size + t.size, dtype=np.uint8)
    qo = q_start + t_start       # q_i after all earlier q's and t's
    to = qo + qlen
    qpos = np.repeat(qo - q_start, qlen) + np.arange(q.size)
    tpos = np.repeat(to - t_start, tlen) + np.arange(t.size)
    arena[qpos] = BASES[q]
    arena[tpos] = BASES[t]
    return PackedPairs.from_arrays(arena, qo.astype(np.uint64), qlen.astype(np.uint32), to.astype(np.uint64),
                                   tlen.astype(np.uint32))


def random_reference(length, seed=0):
    rng = np.random.default_rng(seed)
    return BASES[rng.integers(0, 4, length)].tobytes()


def reads_on_reference(reference, n, length=150, error=0.01, seed=1, sub_frac=0.7, max_indel=3,
                       length_sampler=None):
    """Reads sampled at uniform positions on both strands, mutated at rate `error`.
    Returns (PackedReads, starts, reverse flags)."""
    rng = np.random.default_rng(seed)
    ref = np.frombuffer(reference, dtype=np.uint8)
    codes = np.searchsorted(BASES, ref)
    if length_sampler is None:
        lens = np.full(n, length, dtype=np.int64)
    else:
        lens = np.asarray(length_sampler(rng, n), dtype=np.int64)
    lens = np.minimum(lens, ref.size)
    starts = rng.integers(0, ref.size - lens + 1)
    rev = rng.random(n) < 0.5
    seg_start = np.zeros(n, dtype=np.int64)
    np.cumsum(lens[:-1], out=seg_start[1:])
    idx = np.repeat(starts - seg_start, lens) + np.arange(int(lens.sum()))
    frag = codes[idx].astype(np.uint8)
    mut, mlen = _mutate(rng, frag, seg_start, lens, np.full(n, error), sub_frac=sub_frac, max_indel=max_indel)
    arena = BASES[mut]
    mo = np.zeros(n, dtype=np.int64)
    np.cumsum(mlen[:-1], out=mo[1:])
    reads = []
    for i in range(n):
        r = arena[mo[i]:mo[i] + mlen[i]]
        if rev[i]:
            r = COMP[r[::-1]]
        reads.append(r.tobytes())
    return PackedReads(reads), starts, rev


def extension_pairs_device(n, lo=100, hi=300, max_div=0.05, seed=0, log_uniform=False, max_indel=5, device="cuda"):
    """`extension_pairs` generated on the GPU with torch (same model, its own RNG
    stream): returns a dict of device tensors seq, q_off, q_len, t_off, t_len."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if log_uniform:
        u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
        qlen = torch.exp(np.log(lo) + u * (np.log(hi) - np.log(lo))).long()
    else:
        qlen = torch.randint(lo, hi + 1, (n,), generator=g, device=device)
    qlen = qlen.clamp(lo, hi)
    div = torch.rand(n, generator=g, device=device, dtype=torch.float64) * max_div
    q_start = torch.zeros(n, dtype=torch.long, device=device)
    q_start[1:] = torch.cumsum(qlen, 0)[:-1]
    nq = int(qlen.sum().item())
    q = torch.randint(0, 4, (nq,), generator=g, device=device, dtype=torch.uint8)
    # mutation (see _mutate)
    pair_of = torch.repeat_interleave(torch.arange(n, device=device), qlen)
    ev = torch.rand(nq, generator=g, device=device, dtype=torch.float64) < div[pair_of]
    kind = torch.rand(nq, generator=g, device=device)
    is_sub = ev & (kind < 0.7)
    is_ins = ev & (kind >= 0.7) & (kind < 0.85)
    is_del = ev & (kind >= 0.85)
    klen = torch.randint(1, max_indel + 1, (nq,), generator=g, device=device)
    pos = torch.arange(nq, device=device)
    seg_end = (q_start + qlen)[pair_of]
    del_end = torch.where(is_del, torch.minimum(pos + klen, seg_end), torch.zeros_like(pos))
    run = torch.cummax(del_end, 0).values
    keep = ~(run > pos)
    ins_len = torch.where(is_ins & keep, klen, torch.zeros_like(klen))
    per = keep.long() + ins_len
    out_off = torch.zeros(nq + 1, dtype=torch.long, device=device)
    out_off[1:] = torch.cumsum(per, 0)
    nt = int(out_off[-1].item())
    t = torch.randint(0, 4, (nt,), generator=g, device=device, dtype=torch.uint8)
    shift = torch.randint(1, 4, (nq,), generator=g, device=device, dtype=torch.uint8)
    kept = torch.where(is_sub, (q + shift) % 4, q)
    t[out_off[:-1][keep]] = kept[keep]
    ends = torch.cumsum(qlen, 0)
    tlen = out_off[ends] - out_off[q_start]
    t_start = torch.zeros(n, dtype=torch.long, device=device)
    t_start[1:] = torch.cumsum(tlen, 0)[:-1]
    qo = q_start + t_start
    to = qo + qlen
    bases = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device=device)
    seq = torch.empty(nq + nt + 64, dtype=torch.uint8, device=device)
    seq[torch.repeat_interleave(qo - q_start, qlen) + torch.arange(nq, device=device)] = bases[q.long()]
    seq[torch.repeat_interleave(to - t_start, tlen) + torch.arange(nt, device=device)] = bases[t.long()]
    return {"seq": seq, "q_off": qo.to(torch.uint64), "q_len": qlen.to(torch.uint32),
            "t_off": to.to(torch.uint64), "t_len": tlen.to(torch.uint32), "n": n, "seq_bytes": nq + nt}


def to_packed(d):
    """Host PackedPairs copy of a device pair dict."""
    return PackedPairs.from_arrays(d["seq"][:d["seq_bytes"]].cpu().numpy(), d["q_off"].cpu().numpy(),
                                   d["q_len"].cpu().numpy(), d["t_off"].cpu().numpy(), d["t_len"].cpu().numpy())
