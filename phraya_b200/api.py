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
from .batch import ALN_DTYPE, PackedPairs, PackedReads, READ_RESULT_DTYPE

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

    def __init__(self, device=0, workspace_bytes=0):
        L = lib()
        cfg = A.Config(workspace_bytes, 0, None)
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

    @property
    def kernel_launches(self):
        return int(self._lib.phr_ctx_kernel_launches(self._h))

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
