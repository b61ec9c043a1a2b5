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


def _c_kind(decl):
    """Kind of a C parameter or return type: ptr, i64, i32, u32, f64."""
    d = decl.replace("const", " ").strip()
    if "*" in d:
        return "ptr"
    t = d.split()[0]
    return {"int64_t": "i64", "size_t": "i64", "int32_t": "i32", "int": "i32", "uint32_t": "u32", "double": "f64",
            "homs_status": "i32", "homs_mode": "i32", "homs_memory": "i32", "homs_dtype": "i32"}[t]


def _jl_kind(t):
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{")) or t == "Cstring":
        return "ptr"
    return {"Int64": "i64", "Int32": "i32", "Cint": "i32", "UInt32": "u32", "Cdouble": "f64", "Float64": "f64"}[t]


def header_functions():
    """{name: (return kind, [parameter kinds])} of the header's prototypes."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^([\w ]+?\**)\s*\**\s*(homs_\w+)\(([^;]*?)\);", text, re.M | re.S):
        ret = m.group(1) + ("*" if "*" in text[m.start():m.start(2)] else "")
        params = [p.strip() for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
        kinds = []
        for p in params:
            star = "*" in p
            typ = p.rsplit(None, 1)[0] if not star else p
            kinds.append(_c_kind(typ if not star else "x *"))
        out[m.group(2)] = (_c_kind(ret), kinds)
    return out


def shim_calls():
    """[(name, return kind, [argument kinds])] of every ccall into libhoms in the shim."""
    text = open(SHIM).read()
    out = []
    for m in re.finditer(r"ccall\(\(:(homs_\w+), libhoms\),\s*(\w+),\s*\(([^()]*)\)", text, re.S):
        args = [a for a in (x.strip() for x in m.group(3).split(",")) if a]
        out.append((m.group(1), _jl_kind(m.group(2)), [_jl_kind(a) for a in args]))
    return out


def test_shim_calls_match_the_header():
    # Every ccall of the shim names a function of include/homs.h, with as many
    # arguments as the prototype and of the same kinds (pointer, 64- or 32-bit
    # integer, double), and the same kind of return value.
    hdr = header_functions()
    calls = shim_calls()
    assert len(calls) >= 20
    for name, ret, args in calls:
        assert name in hdr, f"{name} is not declared in include/homs.h"
        c_ret, c_args = hdr[name]
        assert ret == c_ret, (name, ret, c_ret)
        assert args == c_args, (name, args, c_args)
    # and the shim covers the whole-simulation, plan, resident, server, export and builder entry points
    covered = {n for n, _, _ in calls}
    for need in ("homs_simulate", "homs_plan_create", "homs_plan_run", "homs_resident_create",
                 "homs_simulate_resident", "homs_server_create", "homs_server_submit", "homs_server_submit_resident",
                 "homs_server_wait", "homs_server_release", "homs_kspace", "homs_brain_phantom_fill",
                 "homs_csm_birdcage"):
        assert need in covered, need
