"""The C++ host interface (include/dicegpu.hpp) driven from a C++ program,
tests/cpp/schema_driver.cpp, which prints TEST PASSED like the reference's
component-test executables."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def _build():
    subprocess.check_call(["make", "-s", "-C", CPP])
    return os.path.join(CPP, "schema_driver")


def test_cpp_driver_builds_and_links():
    exe = _build()
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_cpp_driver_passes_on_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = _build()
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "TEST PASSED" in out.stdout
