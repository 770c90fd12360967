"""The command line's argument handling on the CPU (warp_peel/__main__.py:13-77):
errors are reported before any device work, with argparse's exit code 2."""

import subprocess
import sys

import pytest
from conftest import ROOT

FIXTURE = ROOT / "tests/golden/fixtures/single.json"


def run(*args):
    return subprocess.run([sys.executable, "-m", "peel_b200", *map(str, args)],
                          capture_output=True, text=True, timeout=300,
                          cwd=ROOT / "exact-depth-peeling_b200")


@pytest.mark.parametrize("args,message", [
    ((FIXTURE,), "--out"),
    ((FIXTURE, "--out", "x.npz", "--method", "clip"), "invalid choice"),
    ((FIXTURE, "--out", "x.npz", "--method", "events", "--pieces", "4", "--device", "cpu"),
     "--pieces applies only to --method peel"),
])
def test_argument_errors(args, message):
    done = run(*args)
    assert done.returncode == 2
    assert message in done.stderr
