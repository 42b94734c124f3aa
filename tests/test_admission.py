"""The request server's admission queue (quoin_b200/csrc/qb_admission.h), on the
CPU: tests/admission_check.cpp is built with g++ and run (budget refusal,
strict arrival order, the budget never exceeded by eight concurrent workers,
close and drain)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_admission_queue(tmp_path):
    exe = str(tmp_path / "admission_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", os.path.join(HERE, "admission_check.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout + r.stderr
