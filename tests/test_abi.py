"""CPU checks of the C ABI: the library loads and exports every declared entry point,
and the ctypes mirror matches the header's struct layouts."""
import ctypes as C
import os
import re

from phraya_b200 import _abi as A
from phraya_b200 import api as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    hdr = open(os.path.join(ROOT, "include", "phraya_gpu.h")).read()
    return sorted(set(re.findall(r"\b(phr_[a-z_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    L = P.lib()
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(A.PROTOTYPES), set(names) ^ set(A.PROTOTYPES)
    assert L.phr_abi_version() == 1


def test_struct_sizes_match_header_layout():
    assert C.sizeof(A.Alignment) == 40
    assert C.sizeof(A.PairBatch) == 72
    assert C.sizeof(A.ReadResult) == 24
    assert C.sizeof(A.Chain) == 24
    assert C.sizeof(A.Seed) == 16
    assert C.sizeof(A.KernelTiming) == 48


def test_no_device_means_engine_unavailable():
    # on a machine without a GPU the context refuses to open (there is no CPU path)
    import torch
    if torch.cuda.is_available():
        return
    try:
        P.Engine(0)
    except P.EngineUnavailable:
        return
    raise AssertionError("Engine opened without a CUDA device")


def test_status_strings():
    L = P.lib()
    for s in range(9):
        assert L.phr_status_string(s)


def test_tune_keys_documented_in_header():
    """Every launch-parameter key phr_ctx_set_tune accepts is documented in the header's
    key list, and every documented key is accepted (read from the sources as text)."""
    with open(os.path.join(ROOT, "phraya_b200", "csrc", "api.cu")) as f:
        src = f.read()
    body = src[src.index("int* tune_field("):src.index("bool tune_valid(")]
    accepted = set(re.findall(r'strcmp\(key, "([a-z_0-9]+)"\)', body))
    with open(os.path.join(ROOT, "include", "phraya_gpu.h")) as f:
        hdr = f.read()
    block = hdr[hdr.index("Launch parameters of the extension kernels"):hdr.index("phr_status phr_ctx_set_tune(")]
    documented = set(re.findall(r'"([a-z_0-9]+)"', block))
    assert accepted and accepted == documented, (accepted ^ documented)


def test_autotuner_keys_are_library_keys():
    """Every key the autotuner searches, and every key it assigns to an engine, is one the
    library accepts (documented in the header's key list)."""
    from phraya_b200 import tune as T
    with open(os.path.join(ROOT, "include", "phraya_gpu.h")) as f:
        hdr = f.read()
    block = hdr[hdr.index("Launch parameters of the extension kernels"):hdr.index("phr_status phr_ctx_set_tune(")]
    documented = set(re.findall(r'"([a-z_0-9]+)"', block))
    assert set(T.SPACE) <= documented
    for keys in T.KEYS_FOR.values():
        assert set(keys) <= set(T.SPACE)
