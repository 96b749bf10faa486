"""The level profiler's command line (the run itself needs a GPU; the profiles cite it)."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_profile_level_help():
    r = subprocess.run([sys.executable, "-m", "curfil_b200.profile_level", "--help"], cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for opt in ("--images", "--features", "--thresholds", "--level", "--tuning"):
        assert opt in r.stdout
