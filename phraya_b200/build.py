"""Builds libphraya_b200.so in-tree with nvcc for sm_100a (B200).

Usage: python -m phraya_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libphraya_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

# the CUDA translation units of the library, one per line; the Rust crate's build.rs
# (rust/phraya-gpu-sys) reads the same list
with open(os.path.join(CSRC, "SOURCES")) as _fh:
    SOURCES = [ln.strip() for ln in _fh if ln.strip() and not ln.startswith("#")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(HERE, "..", "include", "phraya_gpu.h"))
    return files


def sources():
    return [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            sys.stderr.write(f"--- {src}\n{text}")
    if failed:
        msg = "\n".join(f"--- {s}\n{t}" for s, t in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT + ".tmp", *objs,
            "-lcudart", "-lpthread"]
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
