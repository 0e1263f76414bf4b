"""The Fortran interface module (include/pcom_gpu.f90) against the C header
(include/pcom_gpu.h), on the CPU: every bind(c) derived type has the C
struct's members in the same order, at the same byte offsets, with the same
total size, and every interface the module declares is a function the C
header declares and the library exports.

There is no Fortran compiler here, so the module's layout is computed from
its declarations by the interoperability rules of Fortran 2003 (15.3.4):
a bind(c) type lays out like the C struct of the same members, with
c_ptr = 8 bytes, c_int32_t = 4, c_int64_t/c_double = 8, each member aligned
to its own size.  The C side is measured by compiling a small program with
the system C compiler against the header.
"""
import os
import re
import shutil
import subprocess

import pytest

from pcom_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "pcom_gpu.f90")
HDR = os.path.join(ROOT, "include", "pcom_gpu.h")
KIND = {"type(c_ptr)": 8, "integer(c_int32_t)": 4, "integer(c_int64_t)": 8, "real(c_double)": 8,
        "integer(c_int)": 4}


def fortran_types():
    """{type: [(member, elem_size, count)]} from the bind(c) derived types."""
    txt = open(F90).read().lower()
    out = {}
    for m in re.finditer(r"type\s*,\s*bind\(c\)\s*::\s*(\w+)(.*?)end\s+type", txt, re.S):
        name, body = m.group(1), m.group(2)
        mem = []
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            decl, names = line.split("::")
            size = KIND[decl.strip().replace(" ", "")]
            for item in re.findall(r"(\w+)(?:\((\d+)\))?", names):
                mem.append((item[0], size, int(item[1]) if item[1] else 1))
        out[name] = mem
    return out


def fortran_layout(members):
    off, lay = 0, []
    for name, size, count in members:
        off = (off + size - 1) // size * size
        lay.append((name, off))
        off += size * count
    align = max(s for _, s, _ in members)
    return lay, (off + align - 1) // align * align


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    types = fortran_types()
    d = tmp_path_factory.mktemp("abi")
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HDR}"', "int main(void) {"]
    for t, mem in types.items():
        src.append(f'  printf("{t} size %zu\\n", sizeof({t}));')
        for name, _, _ in mem:
            src.append(f'  printf("{t} {name} %zu\\n", offsetof({t}, {name}));')
    src += ["  return 0;", "}"]
    (d / "abi.c").write_text("\n".join(src))
    exe = str(d / "abi")
    subprocess.run([cc, "-std=c11", "-Wall", "-o", exe, str(d / "abi.c")], check=True)
    res = {}
    for line in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        t, m, v = line.split()
        res[(t, m)] = int(v)
    return res


def test_module_declares_every_struct():
    assert set(fortran_types()) == {"pcom_dims", "pcom_static", "pcom_state", "pcom_forcing", "pcom_accum"}


@pytest.mark.parametrize("t", ["pcom_dims", "pcom_static", "pcom_state", "pcom_forcing", "pcom_accum"])
def test_bind_c_layout_matches_header(c_layout, t):
    lay, size = fortran_layout(fortran_types()[t])
    for name, off in lay:
        assert c_layout[(t, name)] == off, f"{t}%{name}: Fortran offset {off}, C offset {c_layout[(t, name)]}"
    assert c_layout[(t, "size")] == size, f"{t}: Fortran size {size}, C size {c_layout[(t, 'size')]}"


def test_c_member_order_matches_module():
    """The header's members, in declaration order, are the module's."""
    hdr = open(HDR).read()
    for t, mem in fortran_types().items():
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (t, t), hdr, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = re.findall(r"\**\s*(\w+)\s*(?:\[\d+\])?\s*[,;]", body)
        assert names == [m[0] for m in mem], t


def test_module_interfaces_are_exported():
    txt = open(F90).read().lower()
    fns = re.findall(r"function\s+(pcom_\w+)\s*\(", txt)
    assert len(fns) >= 15
    lib = L.load()
    for f in fns:
        assert f in L.SIGNATURES, f
        assert hasattr(lib, f), f
