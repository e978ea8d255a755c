"""The gain kernels evaluate the reference's float gain (operatorsDelta.h:29-45, double
divisions rounded to float) through gain_fast: a multiplication by precomputed reciprocals
with a proven error bound, accepted when both ends of the bound round to the same float and
otherwise recomputed with the divisions. This fuzz run compiles tests/gain_fuzz.cu against
the engine's own header and checks gain_fast == gain_exact bit for bit on 2^26 inputs:
generic ones, near cancellation of the two terms, and sums aimed at float rounding
boundaries (where the fallback must take over)."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_gain_fast_equals_divisions(tmp_path):
    exe = str(tmp_path / "gain_fuzz")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-I", os.path.join(ROOT, "louvain-fast-move-cuda_b200", "csrc"),
                    os.path.join(ROOT, "tests", "gain_fuzz.cu"), "-o", exe], check=True)
    p = subprocess.run([exe, "26"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    n, bad, fallbacks = (int(x) for x in p.stdout.split()[:3])
    assert n == 1 << 26 and bad == 0
    # the boundary-aimed inputs must exercise the division fallback
    assert fallbacks > 0
