"""Host logic of the strip SOR's work lists (rgbd-flow_b200/csrc/pipeline.cuh: strip_units,
strip_default_bands, strip_balanced_bands), checked on the CPU.

tests/cpp/strip_units_check.cu includes pipeline.cuh, builds the units of several steps (16 and 1
640x480 pairs, 16 320x240 pairs, the 64-pair mix, ragged sizes) for every band height the
autotuner or an override can ask for and for the balancing model's layouts, and checks that each
band starts on a multiple of 32 rows, that model layouts keep bands of at most 256 rows and cover
their strip, and that the units cover every (item, strip, row) exactly once, largest band first.
It also checks the padded half-row pitch of the register whole-level SOR kernels (level_reg_rp)
and that every cluster shape the plan picks for them fits their 64 KB of shared memory.  No
kernel is launched, so the program runs without a GPU.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc to compile the pipeline header")
def test_strip_units_cover_every_row_once(tmp_path):
    exe = str(tmp_path / "strip_units_check")
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-o", exe,
                    os.path.join(HERE, "cpp", "strip_units_check.cu")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("ok level pitch")
    lines = lines[1:]
    assert len(lines) == 5 * 7 * 2 and all(x.startswith("ok ") for x in lines)
    # the model's layouts of the benchmark's 320x240 step and of the mix's finest step
    assert "ok 16 x 320x240 seg 128 balanced: 320 units H240:32/64/64/80" in lines
    assert any(x.startswith("ok 64-pair mix seg 128 balanced") and "H480:64/192/224" in x for x in lines)
