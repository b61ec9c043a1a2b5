"""The ncu summaries under profiles/ name the commands that made them.

Every summary quotes at least one command, every quoted `python bench.py` /
`python bench_demo.py` command uses only flags those scripts declare (the
subcommand's own flags for bench_demo.py), and nothing points at working
files outside the repository's committed tree."""
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md")))


def _flags(src, holder=r"\w+"):
    return set(re.findall(r"\b" + holder + r"\.add_argument\(\s*\"(--[\w-]+)\"", src))


def _declared():
    bench = open(os.path.join(ROOT, "bench.py")).read()
    demo = open(os.path.join(ROOT, "bench_demo.py")).read()
    subs = {}
    for m in re.finditer(r"(\w+) = sub\.add_parser\(\"(\w+)\"\)", demo):
        subs[m.group(2)] = _flags(demo, m.group(1))
    return _flags(bench, "ap"), subs


def _commands(text):
    return [m.group(0).strip() for m in re.finditer(r"python (?:bench|bench_demo)\.py[^\n`]*", text)]


def test_every_profile_quotes_its_command():
    assert PROFILES
    for path in PROFILES:
        text = open(path).read()
        assert _commands(text), f"{os.path.basename(path)} quotes no command"
        assert "_work/" not in text and "gpurun" not in text, os.path.basename(path)


def test_profile_commands_use_declared_flags():
    bench_flags, demo_subs = _declared()
    assert {"--steps", "--warmup", "--spin-stride", "--no-e2e"} <= bench_flags
    assert set(demo_subs) == {"stage", "run"}
    for path in PROFILES:
        for cmd in _commands(open(path).read()):
            words = cmd.rstrip("\\").split()
            flags = {w for w in words if w.startswith("--")}
            if words[1] == "bench.py":
                unknown = flags - bench_flags
            else:
                unknown = flags - demo_subs[words[2]]
            assert not unknown, (os.path.basename(path), cmd, unknown)
