"""The PML shell decoder (position of a PML cell from its number) and the
multiply-shift division it uses, checked on the CPU against exact division
and a brute-force traversal of the shell.  The kernel header is compiled
with nvcc into a host program (pml_shell_decode_check.cu); no GPU is used."""
import os
import subprocess
import tempfile

import pytest

from ggi_tlm_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shell_decoder_and_fast_division():
    nvcc = build.nvcc()
    if subprocess.run([nvcc, "--version"], capture_output=True).returncode != 0:
        pytest.skip("nvcc not available")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "check")
        cmd = [nvcc, *build.ARCH, "-O2", "-std=c++17", "-o", exe, os.path.join(HERE, "pml_shell_decode_check.cu")]
        res = subprocess.run(cmd, capture_output=True, text=True)
        assert res.returncode == 0, res.stdout + res.stderr
        run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert run.returncode == 0, run.stdout + run.stderr
        assert "fast_div ok, shell ok" in run.stdout
