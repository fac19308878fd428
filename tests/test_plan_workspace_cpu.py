"""The ghost-fill compiler's workspace (kept by a context from one
fx_amr_adapt to the next, together with the retired plan's program arrays)
must not change a plan: tests/plan_workspace_check.cpp compiles a sequence
of meshes of different sizes and kinds (MHD and hydro, uniform and static
AMR) without and with the reused workspace and compares the plans byte for
byte.  Built here with the host compiler from fornaxamr_b200/csrc/fx_plan.cpp;
no GPU is involved."""
import os
import shutil
import subprocess

import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import mesh

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


def _write(tmp_path, name, blocks, coord, mhd):
    prefix = str(tmp_path / name)
    cfg = fx.make_config(mhd, 5.0 / 3.0 if mhd else 1.4, coord)
    with open(prefix + ".cfg", "wb") as f:
        f.write(bytes(cfg))
    with open(prefix + ".desc", "wb") as f:
        f.write(bytes(mesh.to_desc(blocks)))
    return prefix


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC), reason="needs g++ and the CUDA headers")
def test_reused_workspace_gives_the_same_plans(tmp_path):
    exe = str(tmp_path / "plan_workspace_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + CUDA_INC,
                    "-I" + os.path.join(ROOT, "fornaxamr_b200", "csrc"),
                    os.path.join(HERE, "plan_workspace_check.cpp"),
                    os.path.join(ROOT, "fornaxamr_b200", "csrc", "fx_plan.cpp"), "-o", exe],
                   check=True, capture_output=True, timeout=600)
    c = (-0.7, 0.7, -0.7, 0.7, -0.7, 0.7)
    amr3 = _write(tmp_path, "amr3", mesh.static_amr_mesh((3,) * 3, c, 2,
                                                          mesh.ball_refiner((0.1, 0.05, 0.0), (0.4, 0.2))), c, True)
    amr4 = _write(tmp_path, "amr4", mesh.static_amr_mesh((4,) * 3, c, 2,
                                                          mesh.ball_refiner((0.0, 0.0, 0.0), (0.3, 0.15))), c, True)
    uni = _write(tmp_path, "uni", mesh.uniform_mesh((3, 3, 3), c), c, True)
    hyd = _write(tmp_path, "hyd", mesh.static_amr_mesh((2,) * 3, c, 1, mesh.ball_refiner((0.0, 0.0, 0.0), (0.4,))),
                 c, False)
    seq = [amr4, amr3, uni, amr4, hyd, amr3, hyd, amr4]
    r = subprocess.run([exe] + seq, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.split("\n")
    assert sum(1 for l in lines if l.endswith(" same")) == len(seq)
