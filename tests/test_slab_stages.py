"""The batched guard folds: a host harness (tests/slab_stages_check.cu,
built with nvcc, no GPU needed) checks that grouping the slab operations of
the rho and J folds into shared launches changes no result, for every
combination of periodic and open field axes."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not found")
def test_slab_stages_keep_the_fold_results(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "slab_stages_check"
    subprocess.run([nvcc, "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", str(ROOT / "ctca_b200" / "csrc"),
                    str(ROOT / "tests" / "slab_stages_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout
    assert out.stdout.startswith("ok")
