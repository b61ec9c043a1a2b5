"""The Julia drop-in (julia/Homs.jl) against the C ABI, on the CPU.

Julia cannot run here, so the check is mechanical: every `struct` of the shim
names the `include/homs.h` struct it mirrors; its fields must have the C
fields' names, in the same order, at the same byte offsets and sizes, and
the struct the same total size.  The C side comes from a program generated
from the header itself (offsetof / sizeof of every field it declares), so a
change to either file breaks this test."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "homs.h")
SHIM = os.path.join(ROOT, "julia", "Homs.jl")

# Julia isbits field types used by the shim: (size, alignment), x86-64 C layout.
JULIA_TYPES = {"Int64": (8, 8), "UInt64": (8, 8), "Float64": (8, 8), "Cdouble": (8, 8), "Int32": (4, 4),
               "UInt32": (4, 4), "Cint": (4, 4), "Float32": (4, 4), "UInt8": (1, 1), "Int8": (1, 1)}


def _jl_type(t):
    t = t.strip()
    if t.startswith("Ptr{"):
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(.+)\}", t)
    if m:
        size, align = _jl_type(m.group(2))
        return int(m.group(1)) * size, align
    return JULIA_TYPES[t]


def julia_structs():
    """{C struct name: [(field, offset, size)], total size} from the shim."""
    text = open(SHIM).read()
    out = {}
    for m in re.finditer(r"^struct (\w+)\s*# include/homs.h: (\w+)\n(.*?)^end", text, re.M | re.S):
        fields, off, align_max = [], 0, 1
        for line in m.group(3).splitlines():
            line = line.split("#")[0].strip()
            if not line:
                continue
            name, typ = line.split("::", 1)
            size, align = _jl_type(typ)
            off = (off + align - 1) // align * align
            fields.append((name.strip(), off, size))
            off += size
            align_max = max(align_max, align)
        total = (off + align_max - 1) // align_max * align_max
        out[m.group(2)] = (fields, total)
    return out


def header_structs():
    """{C struct name: [field names in order]} parsed from the header."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", text, re.S):
        names = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            first, *rest = decl.split(",")
            declarators = [first.split()[-1]] + [r.strip() for r in rest]
            for d in declarators:
                names.append(re.sub(r"\[.*\]", "", d).lstrip("*").strip())
        out[m.group(1)] = names
    return out


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is not installed")
def test_shim_structs_match_the_header(tmp_path):
    jl = julia_structs()
    hdr = header_structs()
    assert {"homs_phantom", "homs_sequence", "homs_run_options", "homs_state"} <= set(jl)
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "homs.h"', "int main(void) {"]
    for cname in jl:
        assert cname in hdr, f"{cname} is not a struct of include/homs.h"
        lines.append(f'    printf("{cname} SIZE %zu 0\\n", sizeof({cname}));')
        for f in hdr[cname]:
            lines.append(f'    printf("{cname} {f} %zu %zu\\n", offsetof({cname}, {f}), '
                         f'sizeof((({cname} *)0)->{f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    res = subprocess.run(["gcc", "-std=c99", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    c = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, off, size = line.split()
        c.setdefault(s, []).append((f, int(off), int(size)))
    for cname, (fields, total) in jl.items():
        c_fields = [x for x in c[cname] if x[0] != "SIZE"]
        c_total = next(int(x[1]) for x in c[cname] if x[0] == "SIZE")
        assert [f for f, _, _ in fields] == [f for f, _, _ in c_fields], cname
        assert fields == c_fields, (cname, fields, c_fields)
        assert total == c_total, (cname, total, c_total)


def test_a_changed_field_is_caught():
    # The parser sees a type change: HomsRunOptions with a 64-bit method word
    # no longer lays out like homs_run_options.
    fields, total = julia_structs()["homs_run_options"]
    assert fields[0] == ("method", 0, 4) and total == 32
    assert _jl_type("UInt64")[0] != fields[0][2]
