"""The extension microbench at its full size (1,000,000 pairs of 100-300 bp under both
WFA engines, 1,000,000 pairs of 64-2048 bp under global Myers), checked through
size-independent properties of every result rather than against the oracle (which would
take minutes): well-formed CIGARs, consumed spans, edit distance = X + I + D, the whole
query aligned, global spans whole, affine score = the CIGAR's cost. The oracle-exact
tests at smaller sizes are in test_gpu_extend.py."""
import pytest

from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D
from phraya_b200 import validate as V

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full_sets():
    set_a = D.to_packed(D.extension_pairs_device(1_000_000, 100, 300, 0.05, seed=0, device="cuda:0"))
    set_b = D.to_packed(D.extension_pairs_device(1_000_000, 64, 2048, 0.05, seed=1, log_uniform=True,
                                                 device="cuda:0"))
    return set_a, set_b


@pytest.mark.parametrize("engine,costs,which", [(A.ENGINE_WFA_AFFINE, (4, 6, 2), 0),
                                                (A.ENGINE_WFA_LINEAR, (2, 4, 1), 0),
                                                (A.ENGINE_MYERS_GLOBAL, (2, 4, 1), 1)],
                         ids=["wfa_affine", "wfa_linear", "myers_global"])
def test_full_size_results_consistent(full_sets, engine, costs, which):
    p = full_sets[which]
    with P.Engine(0) as eng:
        aln, cig = eng.extend_packed(engine, p, P.AffineCosts(*costs))
    r = V.check_extensions(engine, aln, cig, p.q_len, costs, p.t_len)
    assert r["checked"] == p.n, r  # every pair at 0-5 % divergence aligns
    assert r["violations"] == 0, r
