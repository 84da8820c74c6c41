"""CPU oracle for phraya-align's seed -> chain -> extend path.

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA engine and the timed CPU
baseline. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
package; the product (phraya_b200) never does.

The restatement itself lives in phraya_oracle.cpp (built by the Makefile next to it);
this module is a ctypes wrapper with small pure-Python helpers that tests use to
replay the reference's own seeded fixtures.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from phraya_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force=False):
    """Compiles liboracle.so with the Makefile beside this file."""
    src = os.path.join(_HERE, "phraya_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_lcp.restype = C.c_uint64
        L.orc_lcp.argtypes = [C.c_char_p, C.c_uint64, C.c_char_p, C.c_uint64]
        L.orc_extend_batch.restype = C.c_int32
        L.orc_extend_batch.argtypes = [C.c_int32, C.POINTER(A.PairBatch), A.AffineCosts,
                                       C.POINTER(A.ResultArena), C.c_int32]
        L.orc_extend_batch_time.restype = C.c_uint64
        L.orc_extend_batch_time.argtypes = [C.c_int32, C.POINTER(A.PairBatch), A.AffineCosts, C.c_int32]
        L.orc_sketch.restype = C.c_uint64
        L.orc_sketch.argtypes = [C.c_char_p, C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                 C.c_void_p]
        L.orc_occurrence_cap.restype = C.c_uint64
        L.orc_occurrence_cap.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64]
        L.orc_find_seeds.restype = C.c_uint64
        L.orc_find_seeds.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                     C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64]
        L.orc_chain_seeds.restype = C.c_int64
        L.orc_chain_seeds.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int64, C.c_int64, C.c_uint64,
                                      C.c_uint64, C.c_double, C.c_int64, C.c_void_p, C.c_uint64,
                                      C.c_void_p, C.c_uint64]
        L.orc_score_alignments.restype = C.c_int32
        L.orc_score_alignments.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, C.c_uint64, C.c_void_p,
                                           C.c_void_p]
        L.orc_target_create.restype = C.c_void_p
        L.orc_target_create.argtypes = [C.c_char_p, C.c_uint64, C.c_int32]
        L.orc_target_destroy.restype = None
        L.orc_target_destroy.argtypes = [C.c_void_p]
        L.orc_target_cap.restype = C.c_uint64
        L.orc_target_cap.argtypes = [C.c_void_p]
        L.orc_align_reads.restype = C.c_int32
        L.orc_align_reads.argtypes = [C.c_void_p, C.POINTER(A.ReadBatch), C.POINTER(A.AlignConfig),
                                      C.POINTER(A.ReadResultArena), C.POINTER(A.AlignStats), C.c_int32]
        L.orc_tandem_repeats.restype = C.c_uint64
        L.orc_tandem_repeats.argtypes = [C.c_char_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64]
        L.orc_variants.restype = C.c_int32
        L.orc_variants.argtypes = [C.c_void_p, C.POINTER(A.ReadBatch), C.POINTER(A.ReadResultArena),
                                   C.POINTER(A.AlignConfig), C.POINTER(A.VariantConfig),
                                   C.POINTER(A.VariantArena)]
        L.orc_anchors.restype = C.c_uint64
        L.orc_anchors.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p]
        L.orc_coverage_merge.restype = None
        L.orc_coverage_merge.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int32, C.c_void_p]
        _lib = L
    return _lib


def default_threads():
    return max(1, os.cpu_count() or 1)


from phraya_b200.batch import (PackedPairs, PackedReads, ALN_DTYPE, READ_RESULT_DTYPE,  # noqa: E402
                               VARIANT_DTYPE, ALLELE_DTYPE)


def _unpack_results(n, aln, cig):
    out = []
    for i in range(n):
        a = aln[i]
        s = bytes(cig[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]]).decode()
        out.append((int(a["status"]), s, int(a["edit_distance"]), int(a["query_start"]), int(a["query_end"]),
                    int(a["target_start"]), int(a["target_end"])))
    return out


def extend_packed(engine, packed, costs=(2, 4, 1), nthreads=None):
    """Runs the oracle on a PackedPairs batch; returns (aln ndarray, cigar bytes ndarray)."""
    L = lib()
    aln = np.zeros(packed.n, dtype=ALN_DTYPE)
    cap = packed.cigar_bound()
    cig = np.zeros(cap, dtype=np.uint8)
    arena = A.ResultArena(aln.ctypes.data, cig.ctypes.data, cap, 0)
    b = packed.batch()
    rc = L.orc_extend_batch(engine, C.byref(b), A.AffineCosts(*costs), C.byref(arena),
                            nthreads or default_threads())
    if rc != 0:
        raise RuntimeError(f"orc_extend_batch failed: {rc}")
    return aln, cig[:arena.cigar_used]


def extend(engine, pairs, costs=(2, 4, 1), nthreads=None):
    """Aligns [(q, t[, qseed, tseed]), ...]; returns [(status, cigar, ed, qs, qe, ts, te)]."""
    packed = PackedPairs(pairs)
    aln, cig = extend_packed(engine, packed, costs, nthreads)
    return _unpack_results(packed.n, aln, cig)


def wfa_extend(q, t, qseed=0, tseed=0):
    return extend(A.ENGINE_WFA_LINEAR, [(q, t, qseed, tseed)], nthreads=1)[0]


def wfa_extend_affine(q, t, qseed=0, tseed=0, costs=(2, 4, 1)):
    return extend(A.ENGINE_WFA_AFFINE, [(q, t, qseed, tseed)], costs, nthreads=1)[0]


def myers_extend(q, t, qseed=0, tseed=0):
    return extend(A.ENGINE_MYERS_FIT, [(q, t, qseed, tseed)], nthreads=1)[0]


def myers_edit_distance(q, t):
    r = extend(A.ENGINE_MYERS_GLOBAL, [(q, t)], nthreads=1)[0]
    return r[2], r[1]


def lcp(a, b):
    return int(lib().orc_lcp(bytes(a), len(a), bytes(b), len(b)))


def sketch(seq, k=21, w=11, alphabet=A.ALPHABET_DNA):
    seq = bytes(seq)
    cap = max(len(seq) - k + 1, 0) + 1
    vals = np.zeros(cap, dtype=np.uint64)
    pos = np.zeros(cap, dtype=np.uint32)
    n = lib().orc_sketch(seq, len(seq), k, w, alphabet, vals.ctypes.data, pos.ctypes.data)
    return vals[:n].copy(), pos[:n].copy()


def occurrence_cap(values, positions, floor=256):
    values = np.ascontiguousarray(values, dtype=np.uint64)
    positions = np.ascontiguousarray(positions, dtype=np.uint32)
    return int(lib().orc_occurrence_cap(values.ctypes.data, positions.ctypes.data, len(values), floor))


SEED_DTYPE = np.dtype([("query_pos", "<u4"), ("target_pos", "<u4"), ("minimizer", "<u8")])
CHAIN_DTYPE = np.dtype([("score", "<i8"), ("seed_off", "<u4"), ("n_seeds", "<u4"), ("target_start", "<u4"),
                        ("_pad", "<u4")])


def find_seeds(tvals, tpos, qvals, qpos, max_occ):
    tvals = np.ascontiguousarray(tvals, dtype=np.uint64)
    tpos = np.ascontiguousarray(tpos, dtype=np.uint32)
    qvals = np.ascontiguousarray(qvals, dtype=np.uint64)
    qpos = np.ascontiguousarray(qpos, dtype=np.uint32)
    cap = 1 << 16
    out = np.zeros(cap, dtype=SEED_DTYPE)
    n = lib().orc_find_seeds(tvals.ctypes.data, tpos.ctypes.data, len(tvals), qvals.ctypes.data,
                             qpos.ctypes.data, len(qvals), max_occ, out.ctypes.data, cap)
    return [(int(s["query_pos"]), int(s["target_pos"]), int(s["minimizer"])) for s in out[:n]]


def chain_seeds(seeds, seed_len=21, max_band=100, max_dist_x=100, max_iter=5000, max_skip=25,
                gap_penalty=0.21, min_chain_score=25):
    """seeds: [(qpos, tpos, minimizer)] -> [(score, target_start, [(qpos, tpos, minimizer)])]."""
    arr = np.zeros(max(len(seeds), 1), dtype=SEED_DTYPE)
    for i, (q, t, m) in enumerate(seeds):
        arr[i] = (q, t, m)
    chains = np.zeros(len(seeds) + 1, dtype=CHAIN_DTYPE)
    sout = np.zeros(len(seeds) + 1, dtype=SEED_DTYPE)
    n = lib().orc_chain_seeds(arr.ctypes.data, len(seeds), seed_len, max_band, max_dist_x, max_iter, max_skip,
                              gap_penalty, min_chain_score, chains.ctypes.data, len(chains), sout.ctypes.data,
                              len(sout))
    if n < 0:
        raise RuntimeError("chain buffer too small")
    out = []
    for c in chains[:n]:
        ss = [(int(s["query_pos"]), int(s["target_pos"]), int(s["minimizer"]))
              for s in sout[c["seed_off"]:c["seed_off"] + c["n_seeds"]]]
        out.append((int(c["score"]), int(c["target_start"]), ss))
    return out


def score_alignments(alns, query_len):
    """alns: [(cigar, ed, qs, qe, ts, te)] -> (primary index, [alternative indices])."""
    n = len(alns)
    arr = np.zeros(max(n, 1), dtype=ALN_DTYPE)
    text = b""
    for i, (cig, ed, qs, qe, ts, te) in enumerate(alns):
        arr[i] = (0, ed, qs, qe, ts, te, len(text), len(cig), 0)
        text += cig.encode()
    pi = np.zeros(1, dtype=np.uint64)
    alt = np.zeros(max(n, 1), dtype=np.uint8)
    rc = lib().orc_score_alignments(arr.ctypes.data, text or b"\0", n, query_len, pi.ctypes.data,
                                    alt.ctypes.data)
    if rc != 0:
        raise ValueError("At least one alignment required")
    return int(pi[0]), [i for i in range(n) if alt[i]]


def tandem_repeats(seq):
    """detect_tandem_repeats with min_repeat_count 3 -> [(start, end_inclusive), ...]."""
    seq = bytes(seq)
    cap = max(1, len(seq) // 6 + 1)
    st = np.zeros(cap, dtype=np.uint32)
    en = np.zeros(cap, dtype=np.uint32)
    n = int(lib().orc_tandem_repeats(seq, len(seq), st.ctypes.data, en.ctypes.data, cap))
    assert n <= cap
    return [(int(a), int(b)) for a, b in zip(st[:n], en[:n])]


def anchors(chain_target_starts, strategy):
    """anchors_from_chains: target positions of the anchors (query position 0 each)."""
    st = np.ascontiguousarray(chain_target_starts, dtype=np.uint32)
    out = np.zeros(max(len(st), 1), dtype=np.uint32)
    n = int(lib().orc_anchors(st.ctypes.data if len(st) else None, len(st), strategy, out.ctypes.data))
    return out[:n].tolist()


def coverage_merge(aln, tlen, depth=False, track=None):
    """merge_result's coverage accumulation over an ALN_DTYPE array; returns the track."""
    if track is None:
        track = np.zeros(tlen, dtype=np.uint32)
    aln = np.ascontiguousarray(aln, dtype=ALN_DTYPE)
    lib().orc_coverage_merge(aln.ctypes.data if len(aln) else None, len(aln), tlen, int(depth), track.ctypes.data)
    return track


def variant_config(radius=0, hotspots=()):
    """-> (VariantConfig, keep-alive arrays). hotspots: sorted [(start, end), ...]."""
    hs = np.array([h[0] for h in hotspots], dtype=np.uint32)
    he = np.array([h[1] for h in hotspots], dtype=np.uint32)
    vc = A.VariantConfig(radius, 0, hs.ctypes.data if len(hs) else None, he.ctypes.data if len(he) else None,
                         len(hs))
    return vc, (hs, he)


def unpack_variants(n, off, var, cov, al):
    """-> per read [(position, ref, type, in_repeat, strand, ed, confidence, kmer, coverage list,
    variant_offset, [(allele, count), ...]), ...]"""
    out = []
    for i in range(n):
        rows = []
        for v in var[int(off[i]):int(off[i + 1])]:
            c0 = int(v["coverage_off"])
            a0 = int(v["allele_off"])
            rows.append((int(v["position"]), int(v["ref_base"]), int(v["variant_type"]), int(v["in_tandem_repeat"]),
                         int(v["strand"]), int(v["edit_distance"]), float(v["confidence"]),
                         float(v["kmer_uniqueness"]), cov[c0:c0 + int(v["coverage_len"])].tolist(),
                         int(v["coverage_variant_offset"]),
                         [(int(a["base"]), int(a["count"])) for a in al[a0:a0 + int(v["n_alleles"])]]))
        out.append(rows)
    return out


def unpack_read_results(n, rr, aln, cig):
    """-> [(outcome, has_result, reverse, [(cigar, ed, qs, qe, ts, te), ...])]"""
    out = []
    for i in range(n):
        r = rr[i]
        alns = []
        for j in range(int(r["aln_off"]), int(r["aln_off"]) + int(r["n_aln"])):
            a = aln[j]
            s = bytes(cig[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]]).decode()
            alns.append((s, int(a["edit_distance"]), int(a["query_start"]), int(a["query_end"]),
                         int(a["target_start"]), int(a["target_end"])))
        out.append((int(r["outcome"]), int(r["has_result"]), int(r["reverse"]), alns))
    return out


class Target:
    """TargetContext of the oracle: target bytes + minimizer index + occurrence cap."""

    def __init__(self, target, alphabet=A.ALPHABET_DNA):
        self._t = lib().orc_target_create(bytes(target), len(target), alphabet)
        self.alphabet = alphabet

    def __del__(self):
        if getattr(self, "_t", None):
            lib().orc_target_destroy(self._t)
            self._t = None

    @property
    def cap(self):
        return int(lib().orc_target_cap(self._t))

    def align_packed(self, packed, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, nthreads=None):
        n = packed.n
        rr = np.zeros(n, dtype=READ_RESULT_DTYPE)
        acap = 104 * n + 16
        aln = np.zeros(acap, dtype=ALN_DTYPE)
        ccap = int(acap * 2 * 3 * int(packed.len.max() if n else 1)) + 16
        ccap = min(ccap, 1 << 31)
        cig = np.zeros(ccap, dtype=np.uint8)
        arena = A.ReadResultArena(rr.ctypes.data, aln.ctypes.data, acap, 0, cig.ctypes.data, ccap, 0)
        stats = A.AlignStats()
        cfg = A.AlignConfig(strategy, gap_model)
        b = packed.batch()
        rc = lib().orc_align_reads(self._t, C.byref(b), C.byref(cfg), C.byref(arena), C.byref(stats),
                                   nthreads or default_threads())
        if rc != 0:
            raise RuntimeError(f"orc_align_reads failed: {rc}")
        st = (stats.placed, stats.no_seed, stats.below_threshold, stats.fast_cutoff, stats.no_alignment)
        return rr, aln[:arena.aln_used], cig[:arena.cigar_used], st

    def variants_packed(self, packed, rr, aln, cig, strategy=A.BALANCED, radius=0, hotspots=()):
        """Variant observations (executor.rs:735-775) from align results in phr_align_reads layout.
        Returns (read_variant_off, variants, coverage, alleles) ndarrays."""
        n = packed.n
        off = np.zeros(n + 1, dtype=np.uint64)
        vcap = int(sum(len(bytes(cig[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]])) for a in aln)) + 16
        var = np.zeros(vcap, dtype=VARIANT_DTYPE)
        r = radius or {A.FAST: 150, A.BALANCED: 50}.get(strategy, 25)
        ccap = vcap * (2 * r + 1) + 16
        cov = np.zeros(ccap, dtype=np.uint32)
        acap = int(packed.len.sum()) + vcap + 16
        al = np.zeros(acap, dtype=ALLELE_DTYPE)
        arena = A.VariantArena(off.ctypes.data, var.ctypes.data, vcap, 0, cov.ctypes.data, ccap, 0, al.ctypes.data,
                               acap, 0)
        res = A.ReadResultArena(rr.ctypes.data, aln.ctypes.data, len(aln), len(aln), cig.ctypes.data, len(cig),
                                len(cig))
        vc, keep = variant_config(radius, hotspots)
        cfg = A.AlignConfig(strategy, A.GAP_AFFINE)
        b = packed.batch()
        rc = lib().orc_variants(self._t, C.byref(b), C.byref(res), C.byref(cfg), C.byref(vc), C.byref(arena))
        if rc != 0:
            raise RuntimeError(f"orc_variants failed: {rc}")
        del keep
        return off, var[:arena.variant_used], cov[:arena.coverage_used], al[:arena.allele_used]

    def align_reads(self, reads, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, stored=None, nthreads=None):
        packed = PackedReads(reads, stored)
        rr, aln, cig, st = self.align_packed(packed, strategy, gap_model, nthreads)
        return unpack_read_results(packed.n, rr, aln, cig), st
