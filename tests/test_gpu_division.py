"""The reciprocal-multiplication division used in the broadening filter equals
the correctly rounded device division bit for bit (GPU)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_div_by_grid_is_correctly_rounded(tmp_path):
    exe = str(tmp_path / "div_check")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-ccbin", "/usr/bin/g++", os.path.join(HERE, "cuda", "div_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
