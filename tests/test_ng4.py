"""The four-ghost-layer build runs in its own process (the block layout is
fixed per process by FX_NGHOST): these tests start `pytest` with
FX_NGHOST=4 on tests/ng4_cases.py (device parity of MC and WENO-Z7 against
the PRJ_NGHOST=4 reference builds) and on the ghost-fill compiler tests
(host only), and require them to pass.
"""
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def run_child(args, timeout):
    env = dict(os.environ, FX_NGHOST="4")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider"] + args,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    return r.stdout


def test_ghost_compiler_with_four_ghost_layers():
    out = run_child(["tests/test_mesh_and_ghost_programs.py", "tests/ng4_cases.py", "-m", "not gpu"], 1200)
    assert " passed" in out


@pytest.mark.gpu
def test_device_parity_with_four_ghost_layers():
    out = run_child(["tests/ng4_cases.py", "-m", "gpu"], 1800)
    assert " passed" in out
