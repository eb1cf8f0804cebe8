"""The hand-written adjoint point functions (iflux, Rusanov, boundary ghost
states) against forward-mode dual numbers through the same templated point
physics: <w, J v> = <J^T w, v> to rounding.  Host code compiled by nvcc; no
GPU needed."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not available")
def test_adjoint_point_functions_match_dual_numbers(tmp_path):
    exe = str(tmp_path / "adjoint_points_check")
    src = os.path.join(HERE, "native", "adjoint_points_check.cu")
    subprocess.run([_nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                    "-ffp-contract=off", f"-I{os.path.join(ROOT, 'sddc_b200', 'csrc')}",
                    f"-I{os.path.join(HERE, 'native')}", src, "-o", exe], check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
