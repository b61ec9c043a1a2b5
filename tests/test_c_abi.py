"""The C ABI from plain C: include/homs.h compiles as C99 with -pedantic
-Werror, links against libhoms.so, and its GPU-free calls work."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is not installed")
def test_header_compiles_as_c99_and_links(homs_lib, tmp_path):
    libdir = os.path.join(ROOT, "highordermrisim.jl_b200", "homs")
    exe = tmp_path / "abi_check"
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "c_abi", "abi_check.c"), "-L", libdir, "-lhoms", f"-Wl,-rpath,{libdir}",
           "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    assert "ok" in run.stdout
