"""The drop-in directory on a GPU: callers written the way the reference's own scripts call
`ibp` and `ibp_cuda` (tests/dropin/*.py) run unmodified against the engine with only
dropin/ on PYTHONPATH, and every round trip matches."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(script):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    env = dict(os.environ, PYTHONPATH=os.path.join(REPO, "dropin"))
    r = subprocess.run([sys.executable, os.path.join(REPO, "tests", "dropin", script)],
                       capture_output=True, text=True, env=env, cwd="/", timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if "Match?" in ln]
    return lines, r.stdout


def test_ibp_package_round_trips():
    lines, out = _run("roundtrip_ibp.py")
    assert len(lines) == 6, out
    assert all(ln.endswith("Match? True") for ln in lines), out


def test_ibp_cuda_positional_fetches():
    lines, out = _run("fetch_ibp_cuda.py")
    assert len(lines) == 27, out
    assert all(ln.endswith("Match? True") for ln in lines), out
