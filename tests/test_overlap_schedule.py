"""CPU check of the overlapped reverse sweep's two-stream schedule.

The checkpointed reverse sweep runs its recomputation (advances, stage steps)
on a side stream and its reverse steps on the main stream, renaming checkpoint
slots onto spare buffers so that an advance need not wait for the reverse step
that reads the slot it overwrites (schedule_overlapped in
vortex-transport_b200/csrc/vt_checkpoint.cpp; the GPU runner executes its
output). tests/overlap_schedule_check.cpp replays whole plans on the host: the
adjoint-gradient benchmark's plan (2000 steps, 45 slots), the inverse
problem's (1234 steps, 400 slots) and every plan of up to 40 steps and 6
slots, each with 0, 1 and 2 spare buffers. It checks that every read (advance, stage step, reverse step)
sees the state the sequential plan reads, that each reverse step reads the
stage states of its own step, and that no side-stream write can overtake a
reverse step still reading that buffer or stage-state set.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "vortex-transport_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ is not available")
    exe = str(tmp_path_factory.mktemp("overlap") / "overlap_schedule_check")
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", CSRC,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "overlap_schedule_check.cpp"),
                    os.path.join(CSRC, "vt_checkpoint.cpp"), "-o", exe], check=True)
    return exe


def test_overlapped_schedule_reads_the_sequential_states(checker):
    r = subprocess.run([checker], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK n=2000 S=45" in r.stdout and "OK n=1234 S=400" in r.stdout
    assert r.stdout.strip().splitlines()[-1].startswith("OK all")


@pytest.mark.parametrize("n,S", [(500, 8), (777, 20), (64, 64)])
def test_overlapped_schedule_other_plans(checker, n, S):
    r = subprocess.run([checker, str(n), str(S)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
