"""phraya-io's file formats on the host side: the `.phrayaplan` v7 plan, the
`.phraya.queries` sidecar and the `.phraya` results file.

Encodings restated from phraya-io (no byte of the reference is reused):

* Structs are MessagePack arrays of their fields in declaration order (rmp_serde's
  default, `rmp_serde::to_vec`); maps are MessagePack maps written in ascending key
  order (the reference routes every HashMap through a BTreeMap when serializing,
  plan.rs:10-27, queries.rs:66-96, types.rs:17-23); tuples are arrays; `Option::None`
  is nil; unit enum variants are their (renamed) variant names. A field marked
  `skip_serializing_if` is omitted from the array when empty, so only a trailing group
  of them can be absent (plan.rs:84-96).
* Frames are zstd-compressed at level 3 (`zstd::encode_all(.., 3)`), through the
  system's libzstd.

Plan v7 file (plan.rs:561-660, read side :662-873): "PHR7", the table of contents'
offset as 8 little-endian bytes, the shared frame, one frame per read-sketch chunk, and
the table of contents (uncompressed MessagePack) at that offset.
"""
import ctypes
import ctypes.util
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import msgpack

PHRAYAPLAN_VERSION = 7
PHRAYA_VERSION = 1
V7_MAGIC = b"PHR7"
SCORE_REPORT_THRESHOLD = 0.95

USE_CASES = ("ReadsWithRef", "ReadsOnly", "ContigsWithReads", "ContigsOnly")  # plan.rs:151-162, = 1..4
ALPHABETS = ("Dna", "Protein")                                                 # types.rs:1767-1771
VARIANT_TYPES = ("snp", "insertion", "deletion")                               # types.rs:44-54
STRANDS = ("+", "-")                                                           # types.rs:69-76


class FormatError(ValueError):
    pass


# ---------------------------------------------------------------------------------
# zstd through the system library
# ---------------------------------------------------------------------------------
class _InBuf(ctypes.Structure):
    _fields_ = [("src", ctypes.c_void_p), ("size", ctypes.c_size_t), ("pos", ctypes.c_size_t)]


class _OutBuf(ctypes.Structure):
    _fields_ = [("dst", ctypes.c_void_p), ("size", ctypes.c_size_t), ("pos", ctypes.c_size_t)]


_ZSTD = None


def _zstd():
    global _ZSTD
    if _ZSTD is None:
        name = ctypes.util.find_library("zstd") or "libzstd.so.1"
        z = ctypes.CDLL(name)
        z.ZSTD_compressBound.restype = ctypes.c_size_t
        z.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
        z.ZSTD_compress.restype = ctypes.c_size_t
        z.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        z.ZSTD_isError.restype = ctypes.c_uint
        z.ZSTD_isError.argtypes = [ctypes.c_size_t]
        z.ZSTD_getErrorName.restype = ctypes.c_char_p
        z.ZSTD_getErrorName.argtypes = [ctypes.c_size_t]
        z.ZSTD_createDCtx.restype = ctypes.c_void_p
        z.ZSTD_freeDCtx.argtypes = [ctypes.c_void_p]
        z.ZSTD_decompressStream.restype = ctypes.c_size_t
        z.ZSTD_decompressStream.argtypes = [ctypes.c_void_p, ctypes.POINTER(_OutBuf), ctypes.POINTER(_InBuf)]
        z.ZSTD_DStreamOutSize.restype = ctypes.c_size_t
        _ZSTD = z
    return _ZSTD


def zstd_compress(data: bytes, level: int = 3) -> bytes:
    z = _zstd()
    cap = z.ZSTD_compressBound(len(data))
    out = ctypes.create_string_buffer(cap)
    src = ctypes.create_string_buffer(bytes(data), len(data)) if data else ctypes.create_string_buffer(1)
    n = z.ZSTD_compress(out, cap, src, len(data), level)
    if z.ZSTD_isError(n):
        raise FormatError(f"zstd compression: {z.ZSTD_getErrorName(n).decode()}")
    return out.raw[:n]


def zstd_decompress(data: bytes) -> bytes:
    """Every frame of `data`, decoded by streaming (frames need not carry their size,
    as the Rust zstd crate's streaming writer leaves it out)."""
    z = _zstd()
    dctx = z.ZSTD_createDCtx()
    if not dctx:
        raise FormatError("zstd: no decompression context")
    try:
        src = ctypes.create_string_buffer(bytes(data), len(data)) if data else ctypes.create_string_buffer(1)
        inb = _InBuf(ctypes.cast(src, ctypes.c_void_p), len(data), 0)
        chunk = max(int(z.ZSTD_DStreamOutSize()), 1 << 16)
        buf = ctypes.create_string_buffer(chunk)
        parts = []
        last = 0
        while True:
            outb = _OutBuf(ctypes.cast(buf, ctypes.c_void_p), chunk, 0)
            r = z.ZSTD_decompressStream(dctx, ctypes.byref(outb), ctypes.byref(inb))
            if z.ZSTD_isError(r):
                raise FormatError(f"zstd decompression: {z.ZSTD_getErrorName(r).decode()}")
            parts.append(buf.raw[:outb.pos])
            last = r
            if inb.pos >= inb.size and outb.pos < chunk:
                break
        if last != 0:
            raise FormatError("zstd decompression: truncated frame")
        return b"".join(parts)
    finally:
        z.ZSTD_freeDCtx(dctx)


# ---------------------------------------------------------------------------------
# MessagePack in rmp_serde's shapes
# ---------------------------------------------------------------------------------
def _pack(obj) -> bytes:
    return msgpack.packb(obj, use_bin_type=True)


def _unpack(data: bytes):
    return msgpack.unpackb(data, raw=False, strict_map_key=False, use_list=True)


def _sorted_map(d: dict) -> dict:
    return {k: d[k] for k in sorted(d)}


def _variant(v, names, what):
    """A unit enum variant as written by rmp_serde: its name (also accepted: the variant
    index, or a one-entry map {name: nil})."""
    if isinstance(v, str) and v in names:
        return v
    if isinstance(v, int) and 0 <= v < len(names):
        return names[v]
    if isinstance(v, dict) and len(v) == 1:
        return _variant(next(iter(v)), names, what)
    if isinstance(v, list) and v:
        return _variant(v[0], names, what)
    raise FormatError(f"bad {what}: {v!r}")


def read_content_hash(data: bytes) -> int:
    """FNV-1a 64 of a read's bytes: the key of its stored sketch (plan.rs:29-41)."""
    h = 0xCBF29CE484222325
    for b in data:
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


@dataclass
class Sketch:
    """MinimizerSketch (types.rs:1801-1810): [(value, position)], k, w."""
    minimizers: List[Tuple[int, int]]
    k: int = 21
    w: int = 11

    def to_wire(self):
        return [[int(v), int(p)] for v, p in self.minimizers], int(self.k), int(self.w)

    @classmethod
    def from_wire(cls, x):
        if not isinstance(x, list) or len(x) != 3:
            raise FormatError(f"bad MinimizerSketch: {x!r}")
        return cls([(int(v), int(p)) for v, p in x[0]], int(x[1]), int(x[2]))


@dataclass
class ReferenceSpace:
    """plan.rs:195-205."""
    content_hash: str
    name: Optional[str] = None
    sketches: Dict[str, Sketch] = field(default_factory=dict)


@dataclass
class Plan:
    """PhrayaPlan (plan.rs:262-340) as the v7 reader assembles it."""
    use_case: str = "ReadsWithRef"
    reference_space: List[ReferenceSpace] = field(default_factory=list)
    input_files: List[str] = field(default_factory=list)
    timestamp: str = ""
    kmer_index: Dict[str, Sketch] = field(default_factory=dict)
    kmer_uniqueness: Dict[int, float] = field(default_factory=dict)
    task_list: List[Tuple[int, int]] = field(default_factory=list)
    read_sketches: Dict[int, Sketch] = field(default_factory=dict)
    hotspot_intervals: List[Tuple[int, int]] = field(default_factory=list)
    reads_per_file: List[int] = field(default_factory=list)
    total_read_count: int = 0
    kmer_k: int = 21
    kmer_w: int = 11
    batch_num_chunks: Optional[int] = None
    batch_reads_per_chunk: Optional[int] = None
    read_byte_offsets: List[List[int]] = field(default_factory=list)
    batch_output_paths: List[str] = field(default_factory=list)
    alphabet: str = "Dna"
    insert_size_distribution: Optional[list] = None   # [mean, std_dev, orientation, sample_size]
    mate_info: Dict[str, list] = field(default_factory=dict)   # MateInfo fields as stored
    dense_kmer_index: Dict[str, Sketch] = field(default_factory=dict)
    w11_membership: Dict[str, List[bool]] = field(default_factory=dict)
    sparse_mode: bool = False
    read_hash_order: List[int] = field(default_factory=list)
    version: int = PHRAYAPLAN_VERSION

    def stored_sketch(self, read: bytes):
        """The plan's stored forward sketch of a read, looked up by content hash
        (plan.get_read_sketch, executor.rs:615-624), as (values, positions), or None."""
        sk = self.read_sketches.get(read_content_hash(read))
        if sk is None:
            return None
        return [v for v, _ in sk.minimizers], [p for _, p in sk.minimizers]


# ---------------------------------------------------------------------------------
# Plan v7
# ---------------------------------------------------------------------------------
def _shared_wire(p: Plan):
    """SharedFrame (plan.rs:64-113) in field order."""
    rs = [[r.content_hash, r.name, _sorted_map({k: v.to_wire() for k, v in r.sketches.items()})]
          for r in p.reference_space]
    arr = [PHRAYAPLAN_VERSION, p.use_case, rs, list(p.input_files), p.timestamp,
           _sorted_map({k: v.to_wire() for k, v in p.kmer_index.items()}),
           _sorted_map({int(k): float(v) for k, v in p.kmer_uniqueness.items()}),
           [[int(a), int(b)] for a, b in p.task_list], [[int(a), int(b)] for a, b in p.hotspot_intervals],
           [int(x) for x in p.reads_per_file], int(p.total_read_count), [int(p.kmer_k), int(p.kmer_w)],
           p.batch_num_chunks, p.batch_reads_per_chunk, list(p.batch_output_paths), p.alphabet]
    # the trailing skippable group (plan.rs:96-112); a skipped field shifts every later one
    tail = []
    if p.insert_size_distribution is not None:
        tail.append(list(p.insert_size_distribution))
    if p.dense_kmer_index:
        tail.append(_sorted_map({k: v.to_wire() for k, v in p.dense_kmer_index.items()}))
    if p.w11_membership:
        tail.append(_sorted_map({k: [bool(b) for b in v] for k, v in p.w11_membership.items()}))
    if p.sparse_mode:
        tail.append(True)
    return arr + tail


def _partition(p: Plan, num_chunks: int):
    """partition_read_data (plan.rs:488-559): with a read order, read i's sketch and byte
    offsets go to chunk i / ceil(reads / chunks); without one, everything goes to chunk
    0. Mate information always goes to chunk 0."""
    chunks = [({}, [], {}) for _ in range(num_chunks)]
    if not p.read_hash_order:
        chunks[0] = (dict(p.read_sketches), [list(f) for f in p.read_byte_offsets], dict(p.mate_info))
        return chunks
    total = len(p.read_hash_order)
    size = -(-total // num_chunks) if total else 0
    for pos, h in enumerate(p.read_hash_order):
        c = min(pos // size, num_chunks - 1) if size else 0
        if h in p.read_sketches:
            chunks[c][0][h] = p.read_sketches[h]
    if p.read_byte_offsets:
        for c in range(num_chunks):
            lo, hi = c * size, min((c + 1) * size, total)
            chunks[c] = (chunks[c][0], [list(f[min(lo, len(f)):min(hi, len(f))]) for f in p.read_byte_offsets],
                         chunks[c][2])
    if p.mate_info:
        chunks[0] = (chunks[0][0], chunks[0][1], dict(p.mate_info))
    return chunks


def _chunk_wire(sk, offs, mates):
    arr = [_sorted_map({int(h): s.to_wire() for h, s in sk.items()}), [[int(x) for x in f] for f in offs]]
    if mates:
        arr.append(_sorted_map(dict(mates)))
    return arr


def write_plan(path, plan: Plan):
    """write_plan (plan.rs:561-660): header, shared frame, chunk frames, TOC at the end."""
    n = max(int(plan.batch_num_chunks or 1), 1)
    shared = zstd_compress(_pack(_shared_wire(plan)))
    frames = [zstd_compress(_pack(_chunk_wire(*c))) for c in _partition(plan, n)]
    off = 12 + len(shared)
    table = []
    for f in frames:
        table.append([off, len(f)])
        off += len(f)
    toc = _pack([PHRAYAPLAN_VERSION, 0, n, 12, len(shared), table])
    with open(path, "wb") as fh:
        fh.write(V7_MAGIC)
        fh.write(off.to_bytes(8, "little"))
        fh.write(shared)
        for f in frames:
            fh.write(f)
        fh.write(toc)


def _read_toc(data: bytes):
    """read_toc (plan.rs:662-693)."""
    if len(data) < 12:
        raise FormatError("file too small for v7 header")
    if data[:4] != V7_MAGIC:
        raise FormatError("not a v7 plan file (bad magic)")
    at = int.from_bytes(data[4:12], "little")
    if at > len(data):
        raise FormatError("file truncated: TOC offset past EOF")
    toc = _unpack(data[at:])
    if not isinstance(toc, list) or len(toc) != 6:
        raise FormatError("bad TOC")
    if toc[0] != PHRAYAPLAN_VERSION:
        raise FormatError(f"version mismatch: expected {PHRAYAPLAN_VERSION}, got {toc[0]}")
    return {"version": toc[0], "flags": toc[1], "num_chunks": toc[2], "shared_frame_offset": toc[3],
            "shared_frame_len": toc[4], "chunk_frame_offsets": [tuple(x) for x in toc[5]]}


def read_plan_toc(path):
    with open(path, "rb") as fh:
        return _read_toc(fh.read())


def _frame(data: bytes, off: int, n: int):
    if off + n > len(data):
        raise FormatError("file truncated: frame extends past EOF")
    return _unpack(zstd_decompress(data[off:off + n]))


def _shared_from_wire(a, p: Plan):
    if not isinstance(a, list) or len(a) < 16:
        raise FormatError("bad shared frame")
    p.version = int(a[0])
    p.use_case = _variant(a[1], USE_CASES, "use case")
    p.reference_space = [ReferenceSpace(r[0], r[1], {k: Sketch.from_wire(v) for k, v in r[2].items()})
                         for r in a[2]]
    p.input_files, p.timestamp = list(a[3]), a[4]
    p.kmer_index = {k: Sketch.from_wire(v) for k, v in a[5].items()}
    p.kmer_uniqueness = {int(k): float(v) for k, v in a[6].items()}
    p.task_list = [tuple(x) for x in a[7]]
    p.hotspot_intervals = [tuple(x) for x in a[8]]
    p.reads_per_file, p.total_read_count = list(a[9]), int(a[10])
    p.kmer_k, p.kmer_w = int(a[11][0]), int(a[11][1])
    p.batch_num_chunks, p.batch_reads_per_chunk = a[12], a[13]
    p.batch_output_paths = list(a[14])
    p.alphabet = _variant(a[15], ALPHABETS, "alphabet")
    # trailing skippable group, positional: fill in order, as the reference's reader does
    tail = a[16:]
    if len(tail) > 0:
        p.insert_size_distribution = tail[0]
    if len(tail) > 1:
        p.dense_kmer_index = {k: Sketch.from_wire(v) for k, v in tail[1].items()}
    if len(tail) > 2:
        p.w11_membership = {k: list(v) for k, v in tail[2].items()}
    if len(tail) > 3:
        p.sparse_mode = bool(tail[3])


def read_plan(path, worker: Optional[Tuple[int, int]] = None) -> Plan:
    """read_plan (plan.rs:781-806), or with worker = (id, count) read_plan_worker
    (:808-873) for a pre-split plan (one chunk per worker)."""
    with open(path, "rb") as fh:
        data = fh.read()
    toc = _read_toc(data)
    p = Plan()
    _shared_from_wire(_frame(data, toc["shared_frame_offset"], toc["shared_frame_len"]), p)
    frames = toc["chunk_frame_offsets"]
    if worker is not None:
        wid, wcount = worker
        if toc["num_chunks"] == wcount and wid < len(frames):
            frames = [frames[wid]]
        elif wid < len(frames):
            frames = [frames[wid]]
        else:
            raise FormatError(f"worker_id {wid} exceeds plan chunk count {toc['num_chunks']}")
    for off, n in frames:
        c = _frame(data, off, n)
        if not isinstance(c, list) or len(c) < 2:
            raise FormatError("bad chunk frame")
        hashes = sorted(int(h) for h in c[0])
        p.read_hash_order.extend(hashes)
        for h, s in c[0].items():
            p.read_sketches[int(h)] = Sketch.from_wire(s)
        offs = [list(f) for f in c[1]]
        if offs:
            if not p.read_byte_offsets:
                p.read_byte_offsets = offs
            else:
                for i, f in enumerate(offs):
                    if i < len(p.read_byte_offsets):
                        p.read_byte_offsets[i].extend(f)
        if len(c) > 2:
            p.mate_info.update(c[2])
    return p


# ---------------------------------------------------------------------------------
# .phraya.queries (queries.rs:55-126)
# ---------------------------------------------------------------------------------
def queries_wire(index: Dict[str, List[Tuple[int, float]]]) -> dict:
    """The map write_queries serializes: placements with score >= 0.95, queries left
    with none dropped, positions sorted by (position, score descending), keys ascending."""
    out = {}
    for q in sorted(index):
        kept = [(int(p), float(s)) for p, s in index[q] if s >= SCORE_REPORT_THRESHOLD]
        if not kept:
            continue
        kept.sort(key=lambda x: (x[0], -x[1]))
        out[q] = [[p, s] for p, s in kept]
    return out


def write_queries(path, index: Dict[str, List[Tuple[int, float]]]):
    with open(path, "wb") as fh:
        fh.write(zstd_compress(_pack(queries_wire(index))))


def read_queries(path) -> Dict[str, List[Tuple[int, float]]]:
    with open(path, "rb") as fh:
        m = _unpack(zstd_decompress(fh.read()))
    return {k: [(int(p), float(s)) for p, s in v] for k, v in m.items()}


def query_index(read_ids, read_results) -> Dict[str, List[Tuple[int, float]]]:
    """QueryIndex entries of align_read results (executor.rs:777-781): per read with a
    result, (target_start, 1 - ed / max(|q|, 1)) of the primary and of each alternative.
    read_results are (outcome, has_result, reverse, alignments) rows with alignments
    (cigar, ed, qs, qe, ts, te); the read's length is qe of its primary."""
    out = {}
    for rid, (_, has, _, alns) in zip(read_ids, read_results):
        if not has:
            continue
        qlen = max(alns[0][3], 1)
        out[rid] = [(a[4], 1.0 - a[1] / qlen) for a in alns]
    return out


# ---------------------------------------------------------------------------------
# .phraya (phraya.rs:23-97)
# ---------------------------------------------------------------------------------
@dataclass
class Observation:
    """VariantObservation (types.rs:213-283) in field order."""
    position: int
    ref_base: int
    all_alleles: Dict[int, int]
    confidence: float
    cigar: str
    mapq: int
    edit_distance: int
    local_coverage: List[int]
    avg_base_quality: float
    provenance: str
    in_tandem_repeat: bool = False
    variant_type: str = "snp"
    kmer_uniqueness: float = 1.0
    strand: str = "+"
    total_paired_count: int = 0
    proper_pair_count: int = 0
    insert_size_sum: int = 0
    insert_size_count: int = 0
    coverage_window_variant_offset: int = 0
    mate_info: Optional[list] = None

    def to_wire(self):
        a = [self.position, self.ref_base, _sorted_map({int(k): int(v) for k, v in self.all_alleles.items()}),
             float(self.confidence), self.cigar, self.mapq, self.edit_distance, [int(c) for c in self.local_coverage],
             float(self.avg_base_quality), self.provenance, bool(self.in_tandem_repeat), self.variant_type,
             float(self.kmer_uniqueness), self.strand, self.total_paired_count, self.proper_pair_count,
             self.insert_size_sum, self.insert_size_count, self.coverage_window_variant_offset]
        if self.mate_info is not None:
            a.append(list(self.mate_info))
        return a

    @classmethod
    def from_wire(cls, a):
        if not isinstance(a, list) or len(a) < 10:
            raise FormatError("bad VariantObservation")
        o = cls(int(a[0]), int(a[1]), {int(k): int(v) for k, v in a[2].items()}, float(a[3]), a[4], int(a[5]),
                int(a[6]), list(a[7]), float(a[8]), a[9])
        rest = a[10:]
        names = ("in_tandem_repeat", "variant_type", "kmer_uniqueness", "strand", "total_paired_count",
                 "proper_pair_count", "insert_size_sum", "insert_size_count", "coverage_window_variant_offset",
                 "mate_info")
        for nm, v in zip(names, rest):
            if nm == "variant_type":
                v = _variant(v, VARIANT_TYPES, "variant type")
            elif nm == "strand":
                v = _variant(v, STRANDS, "strand")
            setattr(o, nm, v)
        return o


def coverage_track(coverage) -> Tuple[List[Tuple[int, int]], int]:
    """CoverageTrack::new (types.rs:618-648): per-position counts quantized to the
    nearest 5 ((c + 2) / 5 * 5, at most 255) and run-length encoded."""
    runs = []
    cur, n = 0, 0
    for c in coverage:
        q = min(((int(c) + 2) // 5) * 5, 255)
        if q == cur:
            n += 1
        else:
            if n:
                runs.append((cur, n))
            cur, n = q, 1
    if n:
        runs.append((cur, n))
    return runs, len(coverage)


def write_phraya(path, reference_length, sample_id, timestamp, observations: List[Observation], track):
    """write_phraya (phraya.rs:67-78); `track` is (runs, total_length)."""
    # PhrayaFile = [header, observations, coverage_track]; PhrayaHeader = [version,
    # reference_length, sample_id, timestamp, observation_count]; CoverageTrack = [runs,
    # total_length]
    header = [PHRAYA_VERSION, int(reference_length), sample_id, timestamp, len(observations)]
    runs, total = track
    body = [header, [o.to_wire() for o in observations], [[[int(v), int(n)] for v, n in runs], int(total)]]
    with open(path, "wb") as fh:
        fh.write(zstd_compress(_pack(body)))


def read_phraya(path):
    """read_phraya (phraya.rs:80-97): -> (header dict, observations, (runs, total))."""
    with open(path, "rb") as fh:
        a = _unpack(zstd_decompress(fh.read()))
    if not isinstance(a, list) or len(a) != 3:
        raise FormatError("bad .phraya body")
    h = a[0]
    if h[0] != PHRAYA_VERSION:
        raise FormatError(f"version mismatch: expected {PHRAYA_VERSION}, got {h[0]}")
    header = {"version": h[0], "reference_length": h[1], "sample_id": h[2], "timestamp": h[3],
              "observation_count": h[4]}
    obs = [Observation.from_wire(x) for x in a[1]]
    runs = [(int(v), int(n)) for v, n in a[2][0]]
    return header, obs, (runs, int(a[2][1]))
