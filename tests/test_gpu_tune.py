"""Autotuner: every candidate it tries returns the same (oracle-exact) results, the
tune file round-trips through phr_ctx_create, and out-of-grid values are refused."""
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200 import tune as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("g_short", [1, 2, 4, 8, 16, 32])
def test_group_sizes_bit_exact(g_short):
    """Lanes per short WFA pair off the default still match the oracle."""
    pk = D.extension_pairs(600, 40, 400, 0.08, seed=31)
    with P.Engine(0) as eng:
        eng.set_tune("wfa_group_short", g_short)
        eng.set_tune("wfa_affine_group_short", g_short)
        eng.set_tune("wfa_long_min", 512)
        eng.set_tune("block_threads", 128)
        for engine, costs in ((A.ENGINE_WFA_LINEAR, (2, 4, 1)), (A.ENGINE_WFA_AFFINE, (4, 6, 2))):
            ga, gc = eng.extend_packed(engine, pk, P.AffineCosts(*costs))
            oa, oc = O.extend_packed(engine, pk, costs)
            assert P.unpack(ga, gc) == P.unpack(oa, oc)


def test_tune_and_tune_file(tmp_path):
    wl = T.default_workloads(n_wfa=4000, n_myers=800)
    space = {"wfa_group_short": [8, 16], "block_threads": [128, 256], "myers_band_base": [32, 64],
             "max_blocks_per_sm": [2, 4]}
    with P.Engine(0) as eng:
        start = {k: eng.get_tune(k) for k in space}
        values, ms = T.tune(eng, wl, rounds=1, repeats=1, space=space)
        assert ms > 0
        assert set(values) == {"wfa_group_short", "block_threads", "myers_band_base", "max_blocks_per_sm"}
        for k, v in values.items():
            # a candidate of the space, or the starting value when none beat it
            assert v in space[k] or v == start[k]
        # the engine is left at the chosen values, and they give the oracle's results
        for engine, pk, costs in wl:
            ga, gc = eng.extend_packed(engine, pk, P.AffineCosts(*costs))
            oa, oc = O.extend_packed(engine, pk, costs)
            assert P.unpack(ga, gc) == P.unpack(oa, oc)
    path = tmp_path / "tune.txt"
    T.write_tune_file(str(path), values)
    assert T.read_tune_file(str(path)) == values
    with P.Engine(0, tune_file=str(path)) as e2:
        for k, v in values.items():
            assert e2.get_tune(k) == v


def test_host_chunks_refuses_out_of_range_values():
    with P.Engine(0) as eng:
        for key, bad in (("host_chunks", 1), ("host_chunks", 33)):
            with pytest.raises(P.EngineError):
                eng.set_tune(key, bad)
        eng.set_tune("host_chunks", 8)
        assert eng.get_tune("host_chunks") == 8
