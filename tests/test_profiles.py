"""The ncu summaries under profiles/ each give the command that produced
them; those commands must still run on the committed files.  Every
`python -m crabsaxs_b200.workloads ...` line must parse with the workload
CLI as it is now, and every `python <script>.py` must name a file in the
repository."""
import re
import shlex
from pathlib import Path

import pytest

from crabsaxs_b200 import workloads

ROOT = Path(__file__).resolve().parents[1]
PROFILES = sorted((ROOT / "profiles").glob("*.txt"))


def _commands(text):
    for line in text.splitlines():
        m = re.search(r"python (-m [\w.]+|\S+\.py)(.*?)\s*\\?\s*$", line)
        if m:
            yield m.group(1), shlex.split(m.group(2).split(">")[0])


def test_every_summary_names_its_command():
    assert PROFILES
    for p in PROFILES:
        assert list(_commands(p.read_text())), p.name


@pytest.mark.parametrize("path", PROFILES, ids=lambda p: p.name)
def test_summary_commands_run_on_committed_files(path):
    for target, args in _commands(path.read_text()):
        if target == "-m crabsaxs_b200.workloads":
            ns = workloads.parser().parse_args(args)  # SystemExit on an unknown workload or flag
            assert ns.workload in ("debye-20k", "multipole-100k", "gradient-5k", "pr-100k", "grid-20k")
        elif target.startswith("-m "):
            mod = target[3:].replace(".", "/")
            assert (ROOT / (mod + ".py")).exists() or (ROOT / mod / "__main__.py").exists(), target
        else:
            assert (ROOT / target).is_file(), target
