"""The committed ncu summaries under profiles/: short text files only, each
giving the command that made it; every ncu command there leaves the GPU's
clocks alone (--clock-control none) and runs files that are committed here."""
import os
import re

from conftest import ROOT

PROF = os.path.join(ROOT, "profiles")


def _files():
    return sorted(os.listdir(PROF))


def test_only_short_text_summaries():
    assert _files(), "no profile summaries"
    for f in _files():
        assert f.endswith((".md", ".txt")), f
        assert os.path.getsize(os.path.join(PROF, f)) < 32 * 1024, f


def test_each_ncu_command_keeps_the_clocks_and_runs_committed_files():
    for f in _files():
        text = open(os.path.join(PROF, f)).read()
        blocks = re.findall(r"```\n(.*?)```", text, flags=re.S)
        cmds = [b.replace("\\\n", " ") for b in blocks]
        ncu = [line for b in cmds for line in b.splitlines() if line.strip().startswith("ncu ")]
        assert ncu, f"{f}: no ncu command"
        for line in ncu:
            assert "--clock-control none" in line, (f, line)
        for b in cmds:
            for script in re.findall(r"python (?:-m pytest )?(\S+\.py)", b):
                path = script.split("::")[0]
                assert os.path.exists(os.path.join(ROOT, path)), (f, path)
                assert not path.startswith("_work"), (f, path)
