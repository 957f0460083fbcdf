"""The ncu summaries under profiles/ name commands that still run.

Every summary gives the command that made its figures.  These checks keep
those commands in step with bench.py: each `python bench.py ...` command line
parses with bench.py's own parser (policy overrides included), every `ncu`
command leaves the GPU clocks alone (`--clock-control none`), and the folder
holds text summaries only, naming committed files (no scratch folder, no
home-directory paths).
"""
import glob
import json
import os
import shlex
import sys

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")


def _summaries():
    return sorted(glob.glob(os.path.join(PROFILES, "*")))


def _command_lines(path):
    """The shell command lines of one summary: continuation lines joined,
    trailing comments and markdown backticks dropped."""
    if path.endswith(".json"):
        out = []

        def walk(x):
            if isinstance(x, dict):
                for k, v in x.items():
                    if k == "command" and isinstance(v, str):
                        out.append(v)
                    else:
                        walk(v)
            elif isinstance(x, list):
                for v in x:
                    walk(v)
        walk(json.load(open(path)))
        return out
    lines, cur = [], ""
    for raw in open(path).read().splitlines():
        line = raw.strip()
        if cur:
            line = cur + " " + line
            cur = ""
        if line.endswith("\\"):
            cur = line[:-1].strip()
            continue
        lines.append(line)
    cmds = []
    for line in lines:
        for seg in line.split("`"):
            seg = seg.split("#")[0].strip()
            if seg.startswith(("python bench.py", "ncu ")):
                cmds.append(seg)
    return cmds


def _all_commands():
    return [(os.path.basename(p), c) for p in _summaries() for c in _command_lines(p)]


def test_every_summary_names_its_command():
    for path in _summaries():
        assert _command_lines(path), f"{os.path.basename(path)} gives no command"


def _cases(keep):
    cases = [x for x in _all_commands() if keep(x[1])]
    return dict(argvalues=cases, ids=[f"{n}:{i}" for i, (n, _) in enumerate(cases)])


@pytest.mark.parametrize("name,cmd", **_cases(lambda c: "bench.py" in c))
def test_bench_commands_parse(name, cmd, monkeypatch):
    argv = shlex.split(cmd)
    argv = argv[argv.index("bench.py"):]
    monkeypatch.setattr(sys, "argv", argv)
    a = bench.parse()
    bench.policy_overrides(None, a.policy)  # exits on an unknown knob


@pytest.mark.parametrize("name,cmd", **_cases(lambda c: c.startswith("ncu ") and " -i " not in c))
def test_ncu_commands_leave_the_clocks_alone(name, cmd):
    assert "--clock-control none" in cmd, f"{name}: {cmd}"


def test_profiles_hold_text_summaries_only():
    for path in _summaries():
        assert os.path.splitext(path)[1] in (".md", ".txt", ".json"), path
        text = open(path).read()
        home = os.path.expanduser("~").rstrip("/")
        assert "_work/" not in text, os.path.basename(path)
        assert not home or home + "/" not in text, os.path.basename(path)
