"""The FP64 rho1 work lists on the CPU: tests/cxx/work_list_check.cu is
compiled against the library's internal header and linked against libfrpa.so,
then run without a GPU.  It checks the chunking the host-buffer entry point
overlaps its copies with (ranges of consecutive batches at 6 / 50 / 94 % of the
cost), that the point tiles cover every batch once, and the three work orders."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
LIB_DIR = os.path.join(ROOT, "fast_rpa_eval_b200", "lib")


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not available")
@pytest.mark.skipif(not os.path.exists(os.path.join(LIB_DIR, "libfrpa.so")), reason="libfrpa.so not built")
def test_fp64_work_lists(tmp_path):
    exe = str(tmp_path / "work_list_check")
    build = [NVCC, "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
             "-I" + os.path.join(ROOT, "fast_rpa_eval_b200", "csrc"),
             os.path.join(ROOT, "tests", "cxx", "work_list_check.cu"), "-o", exe,
             "-L" + LIB_DIR, "-lfrpa", "-Xlinker", "-rpath=" + LIB_DIR]
    subprocess.run(build, check=True, capture_output=True, timeout=300)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
