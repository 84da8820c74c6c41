"""Host-side batch packing shared by the engine wrapper and test harnesses.

A batch is a structure of arrays over one byte arena, the layout the C ABI
(include/phraya_gpu.h: phr_pair_batch / phr_read_batch) takes.
"""
import numpy as np

from . import _abi as A

ALN_DTYPE = np.dtype([("status", "<i4"), ("edit_distance", "<u4"), ("query_start", "<u4"),
                      ("query_end", "<u4"), ("target_start", "<u4"), ("target_end", "<u4"),
                      ("cigar_off", "<u8"), ("cigar_len", "<u4"), ("affine_score", "<u4")])

class PackedPairs:
    """Structure-of-arrays pair batch over one byte arena (numpy-owned memory)."""

    def __init__(self, pairs):
        qs, ts, qseed, tseed = [], [], [], []
        for p in pairs:
            q, t = p[0], p[1]
            qs.append(bytes(q))
            ts.append(bytes(t))
            qseed.append(p[2] if len(p) > 2 else 0)
            tseed.append(p[3] if len(p) > 3 else 0)
        n = len(qs)
        q_len = np.array([len(x) for x in qs], dtype=np.uint32)
        t_len = np.array([len(x) for x in ts], dtype=np.uint32)
        arena = b"".join(x for pair in zip(qs, ts) for x in pair)
        offs = np.zeros(2 * n + 1, dtype=np.uint64)
        lens = np.empty(2 * n, dtype=np.uint64)
        lens[0::2] = q_len
        lens[1::2] = t_len
        np.cumsum(lens, out=offs[1:])
        self.seq = np.frombuffer(arena, dtype=np.uint8).copy() if arena else np.zeros(1, np.uint8)
        self.q_off = offs[0:2 * n:2].copy()
        self.t_off = offs[1:2 * n:2].copy()
        self.q_len = q_len
        self.t_len = t_len
        self.q_seed = np.array(qseed, dtype=np.uint32)
        self.t_seed = np.array(tseed, dtype=np.uint32)
        self.n = n

    @classmethod
    def from_arrays(cls, seq, q_off, q_len, t_off, t_len, q_seed=None, t_seed=None):
        self = cls.__new__(cls)
        self.seq, self.q_off, self.q_len, self.t_off, self.t_len = seq, q_off, q_len, t_off, t_len
        self.n = len(q_len)
        self.q_seed = q_seed if q_seed is not None else np.zeros(self.n, np.uint32)
        self.t_seed = t_seed if t_seed is not None else np.zeros(self.n, np.uint32)
        return self

    def batch(self):
        b = A.PairBatch()
        b.n_pairs = self.n
        b.seq = self.seq.ctypes.data
        b.seq_bytes = self.seq.nbytes
        b.q_off = self.q_off.ctypes.data
        b.q_len = self.q_len.ctypes.data
        b.t_off = self.t_off.ctypes.data
        b.t_len = self.t_len.ctypes.data
        b.q_seed = self.q_seed.ctypes.data
        b.t_seed = self.t_seed.ctypes.data
        return b

    def cigar_bound(self):
        return int(2 * (self.q_len.astype(np.uint64).sum() + self.t_len.astype(np.uint64).sum())) + 16


VARIANT_DTYPE = np.dtype([("position", "<u4"), ("ref_base", "u1"), ("variant_type", "u1"),
                          ("in_tandem_repeat", "u1"), ("strand", "u1"), ("read", "<u4"), ("edit_distance", "<u4"),
                          ("confidence", "<f8"), ("kmer_uniqueness", "<f8"), ("coverage_off", "<u8"),
                          ("coverage_len", "<u4"), ("coverage_variant_offset", "<u4"), ("allele_off", "<u8"),
                          ("n_alleles", "<u4"), ("_pad", "<u4")])
assert VARIANT_DTYPE.itemsize == 64

ALLELE_DTYPE = np.dtype([("base", "u1"), ("_pad", "u1", (3,)), ("count", "<u4")])

READ_RESULT_DTYPE = np.dtype([("outcome", "<i4"), ("has_result", "u1"), ("reverse", "u1"), ("_pad", "<u2"),
                              ("n_aln", "<u4"), ("_pad2", "<u4"), ("aln_off", "<u8")])


class PackedReads:
    """Read batch over one byte arena, with optional stored forward sketches."""

    def __init__(self, reads, stored=None):
        reads = [bytes(r) for r in reads]
        self.n = len(reads)
        self.len = np.array([len(r) for r in reads], dtype=np.uint32)
        self.off = np.zeros(self.n, dtype=np.uint64)
        if self.n > 1:
            np.cumsum(self.len[:-1].astype(np.uint64), out=self.off[1:])
        joined = b"".join(reads)
        self.seq = np.frombuffer(joined, dtype=np.uint8).copy() if joined else np.zeros(1, np.uint8)
        self.has_stored = None
        if stored is not None:
            self.has_stored = np.array([1 if s is not None else 0 for s in stored], dtype=np.uint8)
            vals, poss, offs, ns = [], [], [], []
            o = 0
            for s in stored:
                if s is None:
                    offs.append(o)
                    ns.append(0)
                    continue
                v, p = s
                vals.extend(int(x) for x in v)
                poss.extend(int(x) for x in p)
                offs.append(o)
                ns.append(len(v))
                o += len(v)
            self.s_off = np.array(offs, dtype=np.uint64)
            self.s_n = np.array(ns, dtype=np.uint32)
            self.s_values = np.array(vals + [0], dtype=np.uint64)
            self.s_positions = np.array(poss + [0], dtype=np.uint32)

    @classmethod
    def from_arrays(cls, seq, off, lens):
        """Wraps an existing arena (uint8) with per-read offsets (uint64) and lengths (uint32)."""
        self = cls.__new__(cls)
        self.seq = np.ascontiguousarray(seq, dtype=np.uint8) if len(seq) else np.zeros(1, np.uint8)
        self.off = np.ascontiguousarray(off, dtype=np.uint64)
        self.len = np.ascontiguousarray(lens, dtype=np.uint32)
        self.n = len(self.len)
        self.has_stored = None
        return self

    def read(self, i):
        o = int(self.off[i])
        return bytes(self.seq[o:o + int(self.len[i])])

    def subset(self, idx):
        """A new batch holding reads `idx` (in that order)."""
        return PackedReads([self.read(int(i)) for i in idx])

    def batch(self):
        b = A.ReadBatch()
        b.n_reads = self.n
        b.seq = self.seq.ctypes.data
        b.seq_bytes = self.seq.nbytes
        b.off = self.off.ctypes.data
        b.len = self.len.ctypes.data
        if self.has_stored is not None:
            b.has_stored = self.has_stored.ctypes.data
            b.s_off = self.s_off.ctypes.data
            b.s_n = self.s_n.ctypes.data
            b.s_values = self.s_values.ctypes.data
            b.s_positions = self.s_positions.ctypes.data
        return b


