"""Failure paths of the C ABI that are made on the host: a scratch budget too small for
one pair gives that pair PHR_ERR_OOM while the rest of the call is aligned;
bad arguments are refused with PHR_ERR_ARG before any work; a result arena too small
for the CIGAR text gives PHR_ERR_CAPACITY. No kernel is made to fail."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200.batch import PackedPairs

pytestmark = pytest.mark.gpu


def divergent_pair(n, seed):
    rng = np.random.default_rng(seed)
    q = bytes(rng.choice(list(b"ACGT"), n).tolist())
    t = bytes(rng.choice(list(b"ACGT"), n).tolist())
    return q, t


def test_workspace_too_small_is_per_pair_oom():
    """A pair whose extension needs more scratch than the budget reports PHR_ERR_OOM in
    its own status; the other pairs of the call are aligned, and the context goes on."""
    small = D.extension_pairs(64, 100, 300, 0.05, seed=31)
    pairs = [(bytes(small.seq[int(small.q_off[i]):int(small.q_off[i]) + int(small.q_len[i])]),
              bytes(small.seq[int(small.t_off[i]):int(small.t_off[i]) + int(small.t_len[i])])) for i in range(8)]
    with P.Engine(0, workspace_bytes=1 << 20) as eng:
        got = eng.extend(A.ENGINE_WFA_LINEAR, pairs[:4] + [divergent_pair(20000, 1)] + pairs[4:])
        assert got[4][0] == A.PHR_ERR_OOM and got[4][1] == ""
        want = O.extend(A.ENGINE_WFA_LINEAR, pairs)
        assert got[:4] + got[5:] == want
        assert eng.counter("scratch_oom_pairs") == 1
        # the same context still aligns pairs that fit its budget
        ga, gc = eng.extend_packed(A.ENGINE_WFA_AFFINE, small, P.AffineCosts(4, 6, 2))
        oa, oc = O.extend_packed(A.ENGINE_WFA_AFFINE, small, (4, 6, 2))
        assert P.unpack(ga, gc) == P.unpack(oa, oc)


def test_estimates_above_budget_each_get_the_whole_budget():
    """Several long pairs whose first scratch estimate exceeds the budget each get one try
    with the whole budget, in a pass of its own; a pair that fits then is aligned, not
    reported out of memory because an earlier pair took the pass."""
    rng = np.random.default_rng(33)
    pairs = []
    for _ in range(3):
        q = bytearray(rng.choice(list(b"ACGT"), 24000).tolist())
        t = bytearray(q)
        for p in rng.choice(len(t), 120, replace=False):
            t[p] = b"ACGT"[(b"ACGT".index(t[p]) + 1) % 4]
        pairs.append((bytes(q), bytes(t)))
    with P.Engine(0, workspace_bytes=1 << 20) as eng:
        got = eng.extend(A.ENGINE_WFA_LINEAR, pairs)
        assert eng.counter("scratch_oom_pairs") == 0
    assert got == O.extend(A.ENGINE_WFA_LINEAR, pairs)


def test_bad_arguments_are_refused():
    with P.Engine(0) as eng:
        L = eng._lib
        p = PackedPairs([(b"ACGT", b"ACGT")])
        aln = np.zeros(1, dtype=P.ALN_DTYPE)
        cig = np.zeros(16, dtype=np.uint8)
        arena = A.ResultArena(aln.ctypes.data, cig.ctypes.data, 16, 0)
        b = p.batch()
        costs = A.AffineCosts(2, 4, 1)
        assert L.phr_extend_batch(eng.handle, 9, C.byref(b), costs, C.byref(arena)) == A.PHR_ERR_ARG
        assert L.phr_extend_batch(eng.handle, A.ENGINE_MYERS_FIT, None, costs, C.byref(arena)) == A.PHR_ERR_ARG
        assert L.phr_extend_batch(eng.handle, A.ENGINE_MYERS_FIT, C.byref(b), costs, None) == A.PHR_ERR_ARG
        # a pair whose sequence runs past the arena end
        bad = p.batch()
        bad.seq_bytes = 6
        assert L.phr_extend_batch(eng.handle, A.ENGINE_MYERS_FIT, C.byref(bad), costs,
                                  C.byref(arena)) == A.PHR_ERR_ARG
        # the context still works
        assert L.phr_extend_batch(eng.handle, A.ENGINE_MYERS_FIT, C.byref(b), costs, C.byref(arena)) == A.PHR_OK
        assert bytes(cig[:arena.cigar_used]) == b"4M"


def test_cigar_arena_too_small_is_capacity():
    p = D.extension_pairs(50, 100, 300, 0.05, seed=32)
    with P.Engine(0) as eng:
        L = eng._lib
        aln = np.zeros(p.n, dtype=P.ALN_DTYPE)
        cig = np.zeros(8, dtype=np.uint8)
        arena = A.ResultArena(aln.ctypes.data, cig.ctypes.data, 8, 0)
        b = p.batch()
        st = L.phr_extend_batch(eng.handle, A.ENGINE_WFA_LINEAR, C.byref(b), A.AffineCosts(2, 4, 1), C.byref(arena))
        assert st == A.PHR_ERR_CAPACITY
