"""Python mirror of phraya-align's public extension/seeding API over the CUDA engine.

Names, argument meaning and error behaviour follow phraya-align/src/lib.rs:
`wfa_extend`, `wfa_extend_affine`, `myers_extend` return an `Alignment` or raise
`InvalidInput` / `AlignmentFailed` (the two `WfaError` variants, lib.rs:44-49);
`myers_edit_distance` returns `(edit_distance, cigar)`. The batched forms take many
pairs per call -- that is the shape the GPU wants. Every call goes through
libphraya_b200.so (include/phraya_gpu.h); there is no CPU path: if the library or a
CUDA device is missing, calls raise `EngineUnavailable`.
"""
import ctypes as C
import dataclasses
import os
import threading

import numpy as np

from . import _abi as A
from .batch import ALLELE_DTYPE, ALN_DTYPE, PackedPairs, PackedReads, READ_RESULT_DTYPE, VARIANT_DTYPE

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libphraya_b200.so")
_lib = None
_lib_lock = threading.Lock()


class EngineUnavailable(RuntimeError):
    """The CUDA library or a usable device is missing (no CPU fallback exists)."""


class EngineError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


class WfaError(Exception):
    """phraya-align's WfaError (lib.rs:44-49)."""


class InvalidInput(WfaError):
    pass


class AlignmentFailed(WfaError):
    pass


@dataclasses.dataclass(frozen=True)
class SeedAnchor:
    query_pos: int = 0
    target_pos: int = 0


@dataclasses.dataclass(frozen=True)
class Alignment:
    """Alignment (lib.rs:31-39)."""
    cigar: str
    edit_distance: int
    query_start: int
    query_end: int
    target_start: int
    target_end: int


@dataclasses.dataclass(frozen=True)
class AffineCosts:
    """AffineCosts (wfa_simd.rs:521-540); the default is {2, 4, 1}."""
    mismatch: int = 2
    gap_open: int = 4
    gap_extend: int = 1


def lib():
    """Loads libphraya_b200.so (building it first if the sources are newer)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build as _build
                _build.build()
            try:
                _lib = A.bind(C.CDLL(LIB_PATH))
            except OSError as e:
                raise EngineUnavailable(f"cannot load {LIB_PATH}: {e}") from e
    return _lib


class Engine:
    """One device context (phr_ctx): a CUDA stream plus its device workspace."""

    def __init__(self, device=0, workspace_bytes=0, tune_file=None):
        L = lib()
        cfg = A.Config(workspace_bytes, 1 if tune_file else 0, tune_file.encode() if tune_file else None)
        h = C.c_void_p()
        st = L.phr_ctx_create(device, C.byref(cfg), C.byref(h))
        if st != A.PHR_OK:
            raise EngineUnavailable(f"phr_ctx_create failed: {L.phr_status_string(st).decode()}")
        self._h = h
        self._lib = L
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.phr_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, st):
        if st != A.PHR_OK:
            raise EngineError(st, self._lib.phr_ctx_last_error(self._h).decode())

    def set_tune(self, key, value):
        """Sets one kernel launch parameter (phr_ctx_set_tune); results never depend on it."""
        self.check(self._lib.phr_ctx_set_tune(self._h, key.encode(), int(value)))

    def get_tune(self, key):
        v = C.c_int64()
        self.check(self._lib.phr_ctx_get_tune(self._h, key.encode(), C.byref(v)))
        return v.value

    @property
    def kernel_launches(self):
        return int(self._lib.phr_ctx_kernel_launches(self._h))

    def set_timing(self, enable=True):
        """Times every kernel launch with CUDA events (phr_ctx_set_timing)."""
        self.check(self._lib.phr_ctx_set_timing(self._h, 1 if enable else 0))

    def counter(self, name):
        """Work counter of the context (phr_ctx_counter), e.g. "myers_lane_block_columns"."""
        return int(self._lib.phr_ctx_counter(self._h, name.encode()))

    def kernel_times(self):
        """{kernel name: (launches, total ms)} recorded while timing was on."""
        recs = (A.KernelTiming * 64)()
        n = int(self._lib.phr_ctx_get_timing(self._h, recs, 64))
        return {recs[i].name.decode(): (int(recs[i].launches), float(recs[i].total_ms)) for i in range(min(n, 64))}

    # -- pairs API ----------------------------------------------------------
    def extend_packed(self, engine, packed, costs=AffineCosts(), percall=False):
        """Runs one engine over a PackedPairs batch; returns (aln ndarray, cigar bytes)."""
        aln = np.zeros(packed.n, dtype=ALN_DTYPE)
        cap = packed.cigar_bound()
        cig = np.zeros(max(cap, 1), dtype=np.uint8)
        arena = A.ResultArena(aln.ctypes.data, cig.ctypes.data, cap, 0)
        b = packed.batch()
        fn = self._lib.phr_extend_percall if percall else self._lib.phr_extend_batch
        self.check(fn(self._h, engine, C.byref(b), A.AffineCosts(costs.mismatch, costs.gap_open,
                                                                   costs.gap_extend), C.byref(arena)))
        return aln, cig[:arena.cigar_used]

    def extend(self, engine, pairs, costs=AffineCosts()):
        """[(q, t[, qseed, tseed])] -> [(status, cigar, ed, qs, qe, ts, te)]."""
        packed = PackedPairs(pairs)
        aln, cig = self.extend_packed(engine, packed, costs)
        return unpack(aln, cig)


def unpack(aln, cig):
    out = []
    cb = bytes(cig)
    for a in aln:
        s = cb[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]].decode()
        out.append((int(a["status"]), s, int(a["edit_distance"]), int(a["query_start"]), int(a["query_end"]),
                    int(a["target_start"]), int(a["target_end"])))
    return out


_default = None


def default_engine():
    global _default
    if _default is None:
        _default = Engine(0)
    return _default


def _one(engine, query, target, seed, costs=AffineCosts()):
    seed = seed or SeedAnchor()
    r = default_engine().extend(engine, [(bytes(query), bytes(target), seed.query_pos, seed.target_pos)], costs)[0]
    status = r[0]
    if status == A.PHR_INVALID_INPUT:
        raise InvalidInput("Seed position beyond sequence length")
    if status == A.PHR_ALIGNMENT_FAILED:
        raise AlignmentFailed("alignment abandoned: max edit distance exceeded")
    return Alignment(r[1], r[2], r[3], r[4], r[5], r[6])


def wfa_extend(query, target, seed=None):
    """wfa_extend (lib.rs:74)."""
    return _one(A.ENGINE_WFA_LINEAR, query, target, seed)


def wfa_extend_affine(query, target, seed=None, costs=AffineCosts()):
    """wfa_extend_affine (lib.rs:139-167)."""
    return _one(A.ENGINE_WFA_AFFINE, query, target, seed, costs)


def myers_extend(query, target, seed=None):
    """myers_extend (lib.rs:106-127)."""
    return _one(A.ENGINE_MYERS_FIT, query, target, seed)


def myers_edit_distance(query, target):
    """myers_edit_distance (lib.rs:94-96) -> (edit_distance, cigar)."""
    r = default_engine().extend(A.ENGINE_MYERS_GLOBAL, [(bytes(query), bytes(target))])[0]
    return r[2], r[1]


# ---------------------------------------------------------------------------
# Target index, sketching, seeding/chaining and align_read
# ---------------------------------------------------------------------------
class Index:
    """TargetContext on the device (phr_index): target bytes, minimizer index, cap."""

    def __init__(self, engine, target, alphabet=A.ALPHABET_DNA, sketch=None):
        self._eng = engine
        self._lib = engine._lib
        target = bytes(target)
        h = C.c_void_p()
        sk = None
        if sketch is not None:
            vals = np.ascontiguousarray(sketch[0], dtype=np.uint64)
            pos = np.ascontiguousarray(sketch[1], dtype=np.uint32)
            self._keep = (vals, pos)
            sk = A.Sketch(vals.ctypes.data, pos.ctypes.data, len(vals), 0, 0)
        engine.check(self._lib.phr_index_create(engine.handle, target, len(target),
                                                C.byref(sk) if sk is not None else None, alphabet, C.byref(h)))
        self._h = h
        self.alphabet = alphabet
        self.target = target

    @property
    def handle(self):
        return self._h

    def info(self):
        inf = A.IndexInfo()
        self._eng.check(self._lib.phr_index_get_info(self._h, C.byref(inf)))
        return {"n_minimizers": inf.n_minimizers, "n_distinct": inf.n_distinct,
                "occurrence_cap": inf.occurrence_cap, "target_len": inf.target_len,
                "device_bytes": inf.device_bytes}

    def repeat_regions(self):
        """TargetContext::repeat_regions: [(start, end_inclusive), ...] (phr_index_repeat_regions)."""
        n = C.c_uint64(0)
        self._eng.check(self._lib.phr_index_repeat_regions(self._h, None, None, 0, C.byref(n)))
        st = np.zeros(max(n.value, 1), dtype=np.uint32)
        en = np.zeros(max(n.value, 1), dtype=np.uint32)
        self._eng.check(self._lib.phr_index_repeat_regions(self._h, st.ctypes.data, en.ctypes.data, n.value,
                                                           C.byref(n)))
        return [(int(a), int(b)) for a, b in zip(st[:n.value], en[:n.value])]

    def close(self):
        if getattr(self, "_h", None):
            self._lib.phr_index_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _sketch(engine, seqs, k, w, alphabet):
    from .batch import PackedReads
    packed = PackedReads(seqs)
    caps = np.maximum(packed.len.astype(np.int64) - k + 1, 0).astype(np.uint64)
    out_off = np.zeros(packed.n, dtype=np.uint64)
    if packed.n > 1:
        np.cumsum(caps[:-1], out=out_off[1:])
    tot = int(caps.sum()) + 1
    vals = np.zeros(tot, dtype=np.uint64)
    pos = np.zeros(tot, dtype=np.uint32)
    cnt = np.zeros(max(packed.n, 1), dtype=np.uint32)
    sb = A.SeqBatch(packed.n, packed.seq.ctypes.data, packed.seq.nbytes, packed.off.ctypes.data,
                    packed.len.ctypes.data)
    engine.check(engine._lib.phr_sketch_batch(engine.handle, C.byref(sb), k, w, alphabet, out_off.ctypes.data,
                                              vals.ctypes.data, pos.ctypes.data, cnt.ctypes.data))
    return [(vals[o:o + c].copy(), pos[o:o + c].copy()) for o, c in zip(out_off.tolist(), cnt.tolist())]


def _seed_chain(engine, index, sketches):
    n = len(sketches)
    keep = []
    sk = (A.Sketch * max(n, 1))()
    total = 0
    for i, (v, p) in enumerate(sketches):
        v = np.ascontiguousarray(v, dtype=np.uint64)
        p = np.ascontiguousarray(p, dtype=np.uint32)
        keep.append((v, p))
        sk[i] = A.Sketch(v.ctypes.data if len(v) else None, p.ctypes.data if len(p) else None, len(v), 0, 0)
        total += len(v)
    cap = total * int(index.info()["occurrence_cap"]) + 16
    cap = min(cap, 1 << 26)
    nsf = np.zeros(max(n, 1), np.uint32)
    nch = np.zeros(max(n, 1), np.uint32)
    coff = np.zeros(max(n, 1), np.uint64)
    chains = np.zeros(cap, dtype=np.dtype([("score", "<i8"), ("seed_off", "<u4"), ("n_seeds", "<u4"),
                                           ("target_start", "<u4"), ("_pad", "<u4")]))
    seeds = np.zeros(cap, dtype=np.dtype([("query_pos", "<u4"), ("target_pos", "<u4"), ("minimizer", "<u8")]))
    arena = A.ChainArena(nsf.ctypes.data, nch.ctypes.data, coff.ctypes.data, chains.ctypes.data, cap,
                         seeds.ctypes.data, cap)
    engine.check(engine._lib.phr_seed_chain_batch(engine.handle, index.handle, sk, n, C.byref(arena)))
    out = []
    for u in range(n):
        cl = []
        for c in chains[int(coff[u]):int(coff[u]) + int(nch[u])]:
            ss = [(int(s["query_pos"]), int(s["target_pos"]), int(s["minimizer"]))
                  for s in seeds[c["seed_off"]:c["seed_off"] + c["n_seeds"]]]
            cl.append((int(c["score"]), int(c["target_start"]), ss))
        out.append((int(nsf[u]), cl))
    return out


def _align_packed(engine, index, packed, strategy=A.BALANCED, gap_model=A.GAP_AFFINE):
    n = packed.n
    rr = np.zeros(max(n, 1), dtype=READ_RESULT_DTYPE)
    K = 1 if strategy == A.FAST else 2 if strategy == A.BALANCED else 50
    acap = 2 * K * n + 16
    aln = np.empty(acap, dtype=ALN_DTYPE)  # the library writes every entry it reports
    # CIGAR text bound: 6 * len + 16 bytes per alignment of a read of length len
    ccap = 2 * K * (6 * int(packed.len.astype(np.uint64).sum()) + 16 * n) + 64
    cig = np.empty(ccap, dtype=np.uint8)
    arena = A.ReadResultArena(rr.ctypes.data, aln.ctypes.data, acap, 0, cig.ctypes.data, ccap, 0)
    stats = A.AlignStats()
    cfg = A.AlignConfig(strategy, gap_model)
    b = packed.batch()
    engine.check(engine._lib.phr_align_reads(engine.handle, index.handle, C.byref(b), C.byref(cfg), C.byref(arena),
                                             C.byref(stats)))
    st = (stats.placed, stats.no_seed, stats.below_threshold, stats.fast_cutoff, stats.no_alignment)
    return rr[:n], aln[:arena.aln_used], cig[:arena.cigar_used], st


def _align_packed_variants(engine, index, packed, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, radius=0,
                           hotspots=()):
    """phr_align_reads_variants; grows the variant arena once if the first guess is short.
    -> (rr, aln, cig, stats, read_variant_off, variants, coverage, alleles)"""
    n = packed.n
    rr = np.zeros(max(n, 1), dtype=READ_RESULT_DTYPE)
    K = 1 if strategy == A.FAST else 2 if strategy == A.BALANCED else 50
    acap = 2 * K * n + 16
    aln = np.empty(acap, dtype=ALN_DTYPE)
    ccap = 2 * K * (6 * int(packed.len.astype(np.uint64).sum()) + 16 * n) + 64
    cig = np.empty(ccap, dtype=np.uint8)
    hs = np.ascontiguousarray([h[0] for h in hotspots], dtype=np.uint32)
    he = np.ascontiguousarray([h[1] for h in hotspots], dtype=np.uint32)
    vcfg = A.VariantConfig(radius, 0, hs.ctypes.data if len(hs) else None, he.ctypes.data if len(he) else None,
                           len(hs))
    r = radius or (150 if strategy == A.FAST else 50 if strategy == A.BALANCED else 25)
    vcap = max(16, n * 8)
    sizes = [vcap, vcap * (2 * r + 1), vcap * 2]
    off = np.zeros(n + 1, dtype=np.uint64)
    cfg = A.AlignConfig(strategy, gap_model)
    b = packed.batch()
    for _ in range(2):
        var = np.empty(sizes[0], dtype=VARIANT_DTYPE)
        cov = np.empty(sizes[1], dtype=np.uint32)
        al = np.empty(sizes[2], dtype=ALLELE_DTYPE)
        va = A.VariantArena(off.ctypes.data, var.ctypes.data, sizes[0], 0, cov.ctypes.data, sizes[1], 0,
                            al.ctypes.data, sizes[2], 0)
        arena = A.ReadResultArena(rr.ctypes.data, aln.ctypes.data, acap, 0, cig.ctypes.data, ccap, 0)
        stats = A.AlignStats()
        st = engine._lib.phr_align_reads_variants(engine.handle, index.handle, C.byref(b), C.byref(cfg),
                                                  C.byref(arena), C.byref(vcfg), C.byref(va), C.byref(stats))
        if st == A.PHR_ERR_CAPACITY and (va.variant_used > sizes[0] or va.coverage_used > sizes[1]
                                         or va.allele_used > sizes[2]):
            sizes = [max(sizes[0], int(va.variant_used)), max(sizes[1], int(va.coverage_used)),
                     max(sizes[2], int(va.allele_used))]
            continue
        engine.check(st)
        break
    stt = (stats.placed, stats.no_seed, stats.below_threshold, stats.fast_cutoff, stats.no_alignment)
    return (rr[:n], aln[:arena.aln_used], cig[:arena.cigar_used], stt, off, var[:va.variant_used],
            cov[:va.coverage_used], al[:va.allele_used])


def unpack_variants(off, var, cov, al):
    """-> per read [(position, ref, type, in_repeat, strand, ed, confidence, kmer_uniqueness,
    local_coverage, coverage_variant_offset, [(allele, count), ...]), ...]"""
    out = []
    for i in range(len(off) - 1):
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


def unpack_reads(rr, aln, cig):
    """-> [(outcome, has_result, reverse, [(cigar, ed, qs, qe, ts, te), ...])]"""
    out = []
    cb = bytes(cig)
    for r in rr:
        alns = []
        for j in range(int(r["aln_off"]), int(r["aln_off"]) + int(r["n_aln"])):
            a = aln[j]
            s = cb[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]].decode()
            alns.append((s, int(a["edit_distance"]), int(a["query_start"]), int(a["query_end"]),
                         int(a["target_start"]), int(a["target_end"])))
        out.append((int(r["outcome"]), int(r["has_result"]), int(r["reverse"]), alns))
    return out


class CoverageTrack:
    """Device-resident genome coverage track merged batch by batch (phr_coverage_*)."""

    def __init__(self, engine, index, mode=A.COVERAGE_QUANTIZED):
        self._eng = engine
        self._lib = engine._lib
        self.len = int(index.info()["target_len"])
        h = C.c_void_p()
        engine.check(self._lib.phr_coverage_create(engine.handle, index.handle, mode, C.byref(h)))
        self._h = h

    def add(self, aln):
        """Adds the windows of an alignment array (ALN_DTYPE), e.g. align_packed's `aln`."""
        aln = np.ascontiguousarray(aln, dtype=ALN_DTYPE)
        self._eng.check(self._lib.phr_coverage_add(self._h, aln.ctypes.data if len(aln) else None, len(aln)))

    def read(self):
        out = np.zeros(self.len, dtype=np.uint32)
        self._eng.check(self._lib.phr_coverage_read(self._h, out.ctypes.data if self.len else None, self.len))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.phr_coverage_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _engine_index(self, target, alphabet=A.ALPHABET_DNA, sketch=None):
    return Index(self, target, alphabet, sketch)


def _engine_align_reads(self, index, reads, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, stored=None):
    packed = reads if isinstance(reads, PackedReads) else PackedReads(reads, stored)
    rr, aln, cig, st = _align_packed(self, index, packed, strategy, gap_model)
    return unpack_reads(rr, aln, cig), st


def _engine_align_reads_variants(self, index, reads, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, radius=0,
                                 hotspots=(), stored=None):
    """align_read with variant observations: -> (read results, stats, per-read variants)."""
    packed = reads if isinstance(reads, PackedReads) else PackedReads(reads, stored)
    rr, aln, cig, st, off, var, cov, al = _align_packed_variants(self, index, packed, strategy, gap_model, radius,
                                                                 hotspots)
    return unpack_reads(rr, aln, cig), st, unpack_variants(off, var, cov, al)


Engine.index = _engine_index
Engine.coverage_track = lambda self, index, mode=A.COVERAGE_QUANTIZED: CoverageTrack(self, index, mode)
Engine.align_reads_variants = _engine_align_reads_variants
Engine.align_packed_variants = lambda self, index, packed, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, radius=0, \
    hotspots=(): _align_packed_variants(self, index, packed, strategy, gap_model, radius, hotspots)
Engine.align_reads = _engine_align_reads
Engine.align_packed = lambda self, index, packed, strategy=A.BALANCED, gap_model=A.GAP_AFFINE: _align_packed(
    self, index, packed, strategy, gap_model)
Engine.sketch = lambda self, seqs, k=21, w=11, alphabet=A.ALPHABET_DNA: _sketch(self, seqs, k, w, alphabet)
Engine.seed_chain = lambda self, index, sketches: _seed_chain(self, index, sketches)


# ---------------------------------------------------------------------------
# Serving loop (phr_server_*)
# ---------------------------------------------------------------------------
class Server:
    """Continuous-batching read server over a device-resident index."""

    def __init__(self, engine, index, strategy=A.BALANCED, gap_model=A.GAP_AFFINE, max_batch_reads=4096,
                 max_batch_bases=0, max_wait_us=200, n_streams=2, hbm_reserve_bytes=0, short_lane=0,
                 long_blocks_per_sm=0):
        self._eng = engine
        self._lib = engine._lib
        self._index = index
        cfg = A.ServerConfig(A.AlignConfig(strategy, gap_model), max_batch_reads, max_batch_bases, hbm_reserve_bytes,
                             max_wait_us, n_streams, short_lane, long_blocks_per_sm)
        h = C.c_void_p()
        engine.check(self._lib.phr_server_create(engine.handle, index.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        K = 1 if strategy == A.FAST else 2 if strategy == A.BALANCED else 50
        self._K = K
        self._bufs = None

    def submit(self, read):
        rid = C.c_uint64()
        read = bytes(read)
        st = self._lib.phr_server_submit(self._h, read, len(read), C.byref(rid))
        if st != A.PHR_OK:
            raise EngineError(st, "phr_server_submit failed")
        return rid.value

    def submit_many(self, reads):
        """Enqueues several reads in one call; returns their request ids."""
        n = len(reads)
        if n == 0:
            return []
        lens = np.fromiter((len(r) for r in reads), dtype=np.uint32, count=n)
        offs = np.zeros(n, dtype=np.uint64)
        if n > 1:
            np.cumsum(lens[:-1], out=offs[1:])
        seq = b"".join(bytes(r) for r in reads)
        ids = np.zeros(n, dtype=np.uint64)
        st = self._lib.phr_server_submit_many(self._h, seq, offs.ctypes.data, lens.ctypes.data, n, ids.ctypes.data)
        if st != A.PHR_OK:
            raise EngineError(st, "phr_server_submit_many failed")
        return ids.tolist()

    def poll(self, max_results=4096, wait_us=0, max_read_len=100000):
        """Finished requests: [(request_id, (outcome, has_result, reverse, alignments), latency_us)].
        The result buffers are kept across calls; `max_read_len` bounds the CIGAR text of
        one alignment (6 * len + 16 bytes)."""
        acap = max_results * 2 * self._K + 16
        ccap = max_results * self._K * (6 * max_read_len + 16)
        ccap = min(ccap, 1 << 30)
        if self._bufs is None or self._bufs[0] < max_results or self._bufs[2].size < acap or self._bufs[3].size < ccap:
            self._bufs = (max_results, (A.ServerResult * max_results)(), np.empty(acap, dtype=ALN_DTYPE),
                          np.empty(ccap, dtype=np.uint8))
        _, res, aln, cig = self._bufs
        n = C.c_uint32()
        st = self._lib.phr_server_poll(self._h, res, max_results, aln.ctypes.data, aln.size, cig.ctypes.data, cig.size,
                                       wait_us, C.byref(n))
        if st not in (A.PHR_OK,):
            raise EngineError(st, "phr_server_poll failed")
        out = []
        k = 0
        used = 0
        for i in range(n.value):
            k += res[i].n_aln
        if k:
            ends = aln["cigar_off"][:k] + aln["cigar_len"][:k]
            used = int(ends.max())
        cb = cig[:used].tobytes()
        k = 0
        for i in range(n.value):
            r = res[i]
            alns = []
            for _ in range(r.n_aln):
                a = aln[k]
                k += 1
                alns.append((cb[a["cigar_off"]:a["cigar_off"] + a["cigar_len"]].decode(), int(a["edit_distance"]),
                             int(a["query_start"]), int(a["query_end"]), int(a["target_start"]),
                             int(a["target_end"])))
            out.append((int(r.request_id), (int(r.outcome), int(r.has_result), int(r.reverse), alns),
                        float(r.latency_us)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            st = self._lib.phr_server_destroy(self._h)
            self._h = None
            if st != A.PHR_OK:
                raise EngineError(st, "server stopped with an error")

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


Engine.server = lambda self, index, **kw: Server(self, index, **kw)
