"""The C ABI called from C++ (the way a non-Python host binds it): the harness in
tests/harness compiles against include/phraya_gpu.h and links libphraya_b200.so; on the
CPU only the build is checked, on the GPU its output is compared with the oracle."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "harness", "extend_harness.cpp")
LIBDIR = os.path.join(ROOT, "phraya_b200")


def build_harness():
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    from phraya_b200 import build as B
    B.build()
    out = os.path.join(ROOT, "_build", "extend_harness")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    r = subprocess.run([gxx, "-std=c++17", "-O1", SRC, "-o", out, f"-L{LIBDIR}", "-lphraya_b200",
                        f"-Wl,-rpath,{LIBDIR}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def test_harness_builds_and_links():
    exe = build_harness()
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_harness_matches_oracle(tmp_path):
    import oracle as O
    from phraya_b200 import _abi as A
    from phraya_b200 import datagen as D
    exe = build_harness()
    p = D.extension_pairs(300, 100, 300, 0.05, seed=21)
    pairs = [(bytes(p.seq[int(p.q_off[i]):int(p.q_off[i]) + int(p.q_len[i])]),
              bytes(p.seq[int(p.t_off[i]):int(p.t_off[i]) + int(p.t_len[i])])) for i in range(p.n)]
    pairs += [(b"", b"ACGT"), (b"ACGT", b""), (b"ACGTN", b"ACGTN")]
    f = tmp_path / "pairs.txt"
    f.write_text("".join(f"{q.decode() or '-'} {t.decode() or '-'}\n" for q, t in pairs))
    for engine, costs in ((A.ENGINE_WFA_AFFINE, (4, 6, 2)), (A.ENGINE_WFA_LINEAR, (2, 4, 1)),
                          (A.ENGINE_MYERS_FIT, (2, 4, 1)), (A.ENGINE_MYERS_GLOBAL, (2, 4, 1))):
        r = subprocess.run([exe, str(engine), str(f)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        got = [ln.split(" ") for ln in r.stdout.strip("\n").split("\n")]
        want = O.extend(engine, pairs, costs)
        assert len(got) == len(want)
        for g, w in zip(got, want):
            st, ed, qs, qe, ts, te = (int(x) for x in g[:6])
            cig = g[6] if len(g) > 6 else ""
            assert (st, cig, ed, qs, qe, ts, te) == tuple(w[:7]), (engine, g, w)
