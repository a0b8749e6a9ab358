"""The reference's integration tests ported to C++ (tests/cpp/test_correctness.cpp)
through the C++ host API flash-map_b200/include/flash_map.hpp."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "test_correctness")


def test_cpp_api_builds():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "flash-map_b200"), "cpptest"], check=True)
    assert os.path.exists(BIN)


@pytest.mark.gpu
def test_cpp_correctness_port():
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "flash-map_b200"), "cpptest"], check=True)
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok (0 failures)" in r.stdout
