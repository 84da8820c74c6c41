"""GPU parity of the lane-per-pair banded Myers kernel (global engine, 2-bit pairs)
against the CPU oracle, through the C ABI. The band half-width base is swept down to
zero so that many pairs fall outside their first-pass band and take the redo path;
every result must stay bit-exact."""
import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D

pytestmark = pytest.mark.gpu


def _check(eng, packed):
    ga, gc = eng.extend_packed(A.ENGINE_MYERS_GLOBAL, packed)
    oa, oc = O.extend_packed(A.ENGINE_MYERS_GLOBAL, packed, (2, 4, 1))
    g, o = P.unpack(ga, gc), P.unpack(oa, oc)
    bad = [i for i in range(packed.n) if g[i] != o[i]]
    assert not bad, f"{len(bad)}/{packed.n} differ; first #{bad[0]}: gpu={g[bad[0]]} oracle={o[bad[0]]}"


def _indel_heavy(n, seed):
    """Pairs whose lengths differ by up to a third: asymmetric bands."""
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(n):
        L = int(rng.integers(64, 1500))
        q = bytes(rng.choice(list(b"ACGT"), L).tolist())
        t = bytearray(q)
        for _ in range(int(rng.integers(0, 4))):
            p = int(rng.integers(0, len(t)))
            k = int(rng.integers(1, max(2, L // 6)))
            if rng.random() < 0.5:
                del t[p:p + k]
            else:
                t[p:p] = bytes(rng.choice(list(b"ACGT"), k).tolist())
        for _ in range(int(rng.integers(0, L // 40 + 1))):
            t[int(rng.integers(0, len(t)))] = int(rng.choice(list(b"ACGT")))
        pairs.append((q, bytes(t)))
    return O.PackedPairs(pairs)


@pytest.mark.parametrize("ckpt", [1, 0])
@pytest.mark.parametrize("band_base", [64, 16, 0])
def test_lane_kernel_bit_exact_across_bands(band_base, ckpt):
    # ckpt 1: checkpoints every 4 columns and segments recomputed for the traceback;
    # ckpt 0: every column's records stored
    with P.Engine(0) as eng:
        eng.set_tune("myers_lane_ckpt", ckpt)
        eng.set_tune("myers_band_base", band_base)
        eng.set_timing(True)
        _check(eng, D.extension_pairs(2000, 64, 2048, 0.05, seed=31, log_uniform=True))
        _check(eng, _indel_heavy(300, 32))
        times = eng.kernel_times()
        assert times.get("myers_lane", (0, 0.0))[0] >= 2, times


def test_lane_kernel_unrelated_pairs_redo():
    # unrelated sequences: every pair leaves its band and is redone with every block
    rng = np.random.default_rng(33)
    pairs = [(bytes(rng.choice(list(b"ACGT"), L).tolist()), bytes(rng.choice(list(b"ACGT"), L + d).tolist()))
             for L, d in zip(rng.integers(64, 1200, 100), rng.integers(-40, 40, 100))]
    for ckpt in (1, 0):
        with P.Engine(0) as eng:
            eng.set_tune("myers_lane_ckpt", ckpt)
            _check(eng, O.PackedPairs(pairs))


def test_lane_kernel_task_tails_and_tiny_pairs():
    # 1..70 bases (single block), counts that leave partial warps
    rng = np.random.default_rng(34)
    for n in (1, 7, 33, 65):
        pairs = []
        for _ in range(n):
            L = int(rng.integers(1, 70))
            q = bytes(rng.choice(list(b"ACGT"), L).tolist())
            t = bytearray(q)
            for _ in range(int(rng.integers(0, 4))):
                t[int(rng.integers(0, len(t)))] = int(rng.choice(list(b"ACGT")))
            pairs.append((q, bytes(t)))
        for ckpt in (1, 0):
            with P.Engine(0) as eng:
                eng.set_tune("myers_lane_ckpt", ckpt)
                _check(eng, O.PackedPairs(pairs))
