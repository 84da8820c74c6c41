"""GPU test of phr_myers_extend_noalloc, the allocation-free Myers fitting entry point.

That entry point serves callers that cannot allocate device memory themselves (for
example code sharing the GPU with a caching allocator that already holds its memory, or
latency-critical loops that must avoid cudaMalloc/cudaFree and their implicit
synchronisation). Its scratch is one fixed array inside the library, so this test checks
that it returns exactly what the regular batched entry point (phr_extend_batch with
PHR_ENGINE_MYERS_FIT) returns and exactly what the CPU oracle's myers_extend returns, on
two calls in a row that reuse that array, and that pairs beyond its stated length limits
are refused with PHR_ERR_ARG.

The file name sorts last so a run that stops at the first failure has run every other
test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200.batch import PackedPairs

pytestmark = pytest.mark.gpu

MAX_Q, MAX_T, STRIDE = 512, 1024, 3072


def make_pairs(seed):
    rng = np.random.default_rng(seed)
    pairs = []
    ref = D.random_reference(200_000, seed=seed)
    for _ in range(700):  # read-vs-window pairs of the read pipeline (fitting branch)
        s = int(rng.integers(0, len(ref) - 400))
        q = bytearray(ref[s:s + 150])
        for _ in range(int(rng.integers(0, 4))):
            q[int(rng.integers(0, 150))] = int(rng.choice(list(b"ACGT")))
        a = max(0, s - int(rng.integers(0, 3)))
        pairs.append((bytes(q), ref[a:a + 300]))
    for _ in range(300):  # lengths up to the limits, near-equal (global branch) and fitting
        ql = int(rng.integers(1, MAX_Q + 1))
        tl = int(rng.integers(1, MAX_T + 1))
        q = bytes(rng.choice(list(b"ACGT"), ql).tolist())
        t = bytes(rng.choice(list(b"ACGTN"), tl).tolist())
        pairs.append((q, t))
    pairs += [(b"", b"ACGT"), (b"ACGT", b""), (b"A" * MAX_Q, b"A" * MAX_T), (b"ACGTN" * 10, b"ACGTN" * 10)]
    return pairs


def device_batch(torch, packed):
    d = {k: torch.from_numpy(np.ascontiguousarray(getattr(packed, k))).cuda()
         for k in ("seq", "q_off", "q_len", "t_off", "t_len")}
    n = packed.n
    out = {"status": torch.zeros(n, dtype=torch.int32, device="cuda"),
           "ed": torch.zeros(n, dtype=torch.int32, device="cuda"),
           "consumed": torch.zeros(n, dtype=torch.int32, device="cuda"),
           "cigar": torch.zeros(n * STRIDE, dtype=torch.uint8, device="cuda"),
           "cigar_len": torch.zeros(n, dtype=torch.int32, device="cuda")}
    return d, out


def run_noalloc(L, torch, d, out, n):
    return L.phr_myers_extend_noalloc(d["seq"].data_ptr(), d["q_off"].data_ptr(), d["q_len"].data_ptr(),
                                      d["t_off"].data_ptr(), d["t_len"].data_ptr(), n, out["status"].data_ptr(),
                                      out["ed"].data_ptr(), out["consumed"].data_ptr(), out["cigar"].data_ptr(),
                                      STRIDE, out["cigar_len"].data_ptr(), None)


def results(out, n):
    st = out["status"].cpu().numpy()
    ed = out["ed"].cpu().numpy()
    cons = out["consumed"].cpu().numpy()
    cl = out["cigar_len"].cpu().numpy()
    cig = out["cigar"].cpu().numpy().tobytes()
    return [(int(st[i]), cig[i * STRIDE:i * STRIDE + int(cl[i])].decode(), int(ed[i]), int(cons[i]))
            for i in range(n)]


def test_noalloc_matches_batched_entry_point_twice():
    torch = pytest.importorskip("torch")
    eng = P.Engine(0)
    L = eng._lib
    for seed in (1, 2):  # two calls in a row over the shared scratch array
        packed = PackedPairs(make_pairs(seed))
        aln, cig = eng.extend_packed(A.ENGINE_MYERS_FIT, packed)
        ref = [(r[0], r[1], r[2], r[6] - r[5]) for r in P.unpack(aln, cig)]
        oa, oc = O.extend_packed(A.ENGINE_MYERS_FIT, packed, (2, 4, 1))
        orc = [(r[0], r[1], r[2], r[6] - r[5]) for r in P.unpack(oa, oc)]
        d, out = device_batch(torch, packed)
        assert run_noalloc(L, torch, d, out, packed.n) == A.PHR_OK
        got = results(out, packed.n)
        bad = [i for i in range(packed.n) if got[i] != ref[i]]
        assert not bad, (len(bad), got[bad[0]], ref[bad[0]])
        bad = [i for i in range(packed.n) if got[i] != orc[i]]
        assert not bad, (len(bad), got[bad[0]], orc[bad[0]])
    eng.close()


def test_noalloc_rejects_pairs_beyond_limits():
    torch = pytest.importorskip("torch")
    L = P.lib()
    torch.cuda.init()
    packed = PackedPairs([(b"ACGT" * 20, b"ACGT" * 30), (b"A" * (MAX_Q + 1), b"A" * 600),
                          (b"ACGT", b"C" * (MAX_T + 1))])
    d, out = device_batch(torch, packed)
    assert run_noalloc(L, torch, d, out, packed.n) == A.PHR_ERR_ARG
    st = out["status"].cpu().numpy().tolist()
    assert st == [A.PHR_OK, A.PHR_ERR_ARG, A.PHR_ERR_ARG]
    # a stride below the stated minimum is refused before any work
    assert L.phr_myers_extend_noalloc(d["seq"].data_ptr(), d["q_off"].data_ptr(), d["q_len"].data_ptr(),
                                      d["t_off"].data_ptr(), d["t_len"].data_ptr(), packed.n,
                                      out["status"].data_ptr(), out["ed"].data_ptr(), out["consumed"].data_ptr(),
                                      out["cigar"].data_ptr(), STRIDE - 1, out["cigar_len"].data_ptr(),
                                      None) == A.PHR_ERR_ARG
