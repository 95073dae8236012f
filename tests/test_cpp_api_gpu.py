"""Runs the C++ program that exercises the linalg_backend::B200 operator
specializations through the reference's own template API (GPU)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu


def test_cpp_operator_api():
    from linearalgebra_b200 import build as b
    exe = b.CPP_TEST_BIN
    if not os.path.exists(exe):
        exe = b.build_cpp_test()
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "ALL PASSED" in res.stdout
