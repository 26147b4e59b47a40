"""The library from plain C, as the reference's own callers use it: the
program in tests/c/ (the flow of the reference's tests/testing_zposv.c, plus
ScaLAPACK's PDPOTRF) is compiled against include/dplasma_b200.h and linked
against the shared library with gcc.  CPU: it compiles and links warning-free.
GPU: it runs and both of the reference's residual ratios are below 10."""
import os
import subprocess

import pytest

import dplasma_b200 as db

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "dposv_tester.c")


def build(tmp_path):
    lib_dir = os.path.dirname(db.lib()._name)
    exe = str(tmp_path / "dposv_tester")
    cmd = ["gcc", "-O2", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + lib_dir, "-ldplasma_b200", "-Wl,-rpath," + lib_dir, "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_c_caller_dposv_and_pdpotrf(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe, "1000", "256", "8"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "ok" in r.stdout.split(), r.stdout
    r = subprocess.run([exe, "700", "93", "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
