"""Host batches large enough to run in overlapped chunks (phr_extend_batch) must give
exactly the results of the device-resident call (phr_extend_batch_device) on the same
pairs: same alignment records (CIGAR offsets included) and the same packed CIGAR text."""
import ctypes as C

import numpy as np
import pytest

from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D

pytestmark = pytest.mark.gpu


def _device_call(eng, engine, packed, costs):
    import torch
    dev = {k: torch.from_numpy(np.ascontiguousarray(getattr(packed, k))).cuda()
           for k in ("seq", "q_off", "q_len", "t_off", "t_len", "q_seed", "t_seed")}
    b = A.PairBatch()
    b.n_pairs = packed.n
    b.seq, b.seq_bytes = dev["seq"].data_ptr(), packed.seq.nbytes
    b.q_off, b.q_len = dev["q_off"].data_ptr(), dev["q_len"].data_ptr()
    b.t_off, b.t_len = dev["t_off"].data_ptr(), dev["t_len"].data_ptr()
    b.q_seed, b.t_seed = dev["q_seed"].data_ptr(), dev["t_seed"].data_ptr()
    cap = packed.cigar_bound()
    aln = torch.empty(packed.n * C.sizeof(A.Alignment), dtype=torch.uint8, device="cuda")
    cig = torch.empty(cap, dtype=torch.uint8, device="cuda")
    arena = A.ResultArena(aln.data_ptr(), cig.data_ptr(), cap, 0)
    eng.check(eng._lib.phr_extend_batch_device(eng.handle, engine, C.byref(b), A.AffineCosts(*costs),
                                               C.byref(arena)))
    torch.cuda.synchronize()
    return aln.cpu().numpy().view(P.ALN_DTYPE), bytes(cig[:arena.cigar_used].cpu().numpy())


@pytest.mark.parametrize("engine,costs", [(A.ENGINE_WFA_AFFINE, (4, 6, 2)), (A.ENGINE_MYERS_GLOBAL, (2, 4, 1))],
                         ids=["affine", "myers_global"])
def test_chunked_host_batch_equals_device_call(engine, costs):
    packed = D.to_packed(D.extension_pairs_device(450_000, 100, 300, 0.05, seed=41))
    rng = np.random.default_rng(42)
    # nonzero seeds on some pairs exercise the seed-array copies of every chunk
    packed.q_seed = np.where(rng.random(packed.n) < 0.1, rng.integers(0, 50, packed.n), 0).astype(np.uint32)
    packed.t_seed = np.minimum(packed.q_seed, packed.t_len).astype(np.uint32)
    assert packed.seq.nbytes > (128 << 20)  # large enough to be split into chunks
    with P.Engine(0) as eng:
        ha, hc = eng.extend_packed(engine, packed, P.AffineCosts(*costs))
        da, dc = _device_call(eng, engine, packed, costs)
    assert np.array_equal(ha, da)
    assert bytes(hc) == dc


@pytest.mark.parametrize("chunks", [2, 16])
def test_chunk_count_does_not_change_results(chunks):
    """host_chunks only changes how a host batch is split and overlapped."""
    packed = D.to_packed(D.extension_pairs_device(450_000, 100, 300, 0.05, seed=43))
    with P.Engine(0) as eng:
        eng.set_tune("host_chunks", chunks)
        ha, hc = eng.extend_packed(A.ENGINE_WFA_LINEAR, packed, P.AffineCosts(2, 4, 1))
        da, dc = _device_call(eng, A.ENGINE_WFA_LINEAR, packed, (2, 4, 1))
    assert np.array_equal(ha, da)
    assert bytes(hc) == dc
