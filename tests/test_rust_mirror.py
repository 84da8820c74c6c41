"""The Rust FFI crate (rust/phraya-gpu-sys) against the C header, on the CPU.

Rust is not installed here, so the crate is checked by what it declares: every
`#[repr(C)]` struct's size and field offsets (computed from the Rust field types with
C layout rules) are turned into static_asserts over the header's structs and compiled
with g++; every function of the header is declared in the crate's extern block with
the same number of parameters; the crate's build script reads the same CUDA source
manifest as the Python build.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_RS = os.path.join(ROOT, "rust", "phraya-gpu-sys", "src", "lib.rs")
HEADER = os.path.join(ROOT, "include", "phraya_gpu.h")

PRIM = {"u8": (1, 1), "i8": (1, 1), "u16": (2, 2), "i16": (2, 2), "u32": (4, 4), "i32": (4, 4), "f32": (4, 4),
        "u64": (8, 8), "i64": (8, 8), "f64": (8, 8), "c_char": (1, 1), "usize": (8, 8)}


def rust_structs():
    src = open(LIB_RS).read()
    out = {}
    for m in re.finditer(r"#\[repr\(C\)\]\s*(?:#\[derive\([^)]*\)\]\s*)?pub struct (\w+) \{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        fields = re.findall(r"(?:pub )?(\w+):\s*([^,\n]+),", body)
        out[name] = [(f, t.strip()) for f, t in fields]
    return out


def layout(structs, name):
    """(size, align, [(field, offset)]) of a repr(C) struct."""
    off, align, rows = 0, 1, []
    for f, t in structs[name]:
        if t.startswith("*"):
            sz, al = 8, 8
        elif t.startswith("["):
            inner, count = re.match(r"\[(\w+);\s*(\d+)\]", t).groups()
            isz, al = PRIM[inner]
            sz = isz * int(count)
        elif t in PRIM:
            sz, al = PRIM[t]
        else:
            sz, al, _ = layout(structs, t)
        off = (off + al - 1) // al * al
        rows.append((f, off))
        off += sz
        align = max(align, al)
    size = (off + align - 1) // align * align
    return size, align, rows


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"^[\w \*]+?\b(phr_\w+)\s*\(([^;{]*?)\);", src, re.M | re.S):
        args = m.group(2).strip()
        n = 0 if args in ("", "void") else args.count(",") + 1
        out[m.group(1)] = n
    return out


def rust_functions():
    src = open(LIB_RS).read()
    block = re.search(r'extern "C" \{(.*?)\n\}', src, re.S).group(1)
    out = {}
    for m in re.finditer(r"pub fn (\w+)\((.*?)\)", block, re.S):
        args = m.group(2).strip().rstrip(",")
        out[m.group(1)] = 0 if not args else args.count(",") + 1
    return out


def test_every_header_function_is_bound():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 30
    assert set(h) == set(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    for name, n in h.items():
        assert r[name] == n, (name, n, r[name])


def test_struct_layouts_match_header():
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    structs = rust_structs()
    opaque = {"phr_ctx", "phr_index", "phr_coverage", "phr_server"}
    lines = ["#include <cstddef>", f'#include "{HEADER}"']
    checked = 0
    for name in structs:
        if name in opaque:
            continue
        size, _, rows = layout(structs, name)
        lines.append(f'static_assert(sizeof({name}) == {size}, "{name} size");')
        for f, off in rows:
            lines.append(f'static_assert(offsetof({name}, {f}) == {off}, "{name}.{f}");')
        checked += 1
    assert checked >= 20
    work = os.path.join(ROOT, "_build")
    os.makedirs(work, exist_ok=True)
    cpp = os.path.join(work, "rust_mirror_layout.cpp")
    with open(cpp, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", cpp], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_build_script_reads_the_shared_source_manifest():
    from phraya_b200 import build as B
    rs = open(os.path.join(ROOT, "rust", "phraya-gpu-sys", "build.rs")).read()
    assert '"SOURCES"' in rs
    listed = [ln.strip() for ln in open(os.path.join(ROOT, "phraya_b200", "csrc", "SOURCES")) if ln.strip()]
    assert listed == B.SOURCES
    on_disk = sorted(f for f in os.listdir(os.path.join(ROOT, "phraya_b200", "csrc")) if f.endswith(".cu"))
    assert sorted(listed) == on_disk
