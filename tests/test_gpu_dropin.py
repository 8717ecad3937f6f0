"""The reference's test suite restated in C++ (tests/cpp/test_dropin.cpp) against the drop-in classes with the
reference's names and signatures (molecular-dynamics_b200/dropin), which run on the GPU. Includes the
md_sim config-1 state hashes after 1 and 1000 steps through the C++ API."""
from __future__ import annotations

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "test_dropin")

pytestmark = pytest.mark.gpu


def test_dropin_cpp_suite(md):
    subprocess.run(["make", "--no-print-directory", "-C", os.path.join(ROOT, "molecular-dynamics_b200", "dropin")],
                   check=True)
    subprocess.run(["make", "--no-print-directory", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=900)
    print(r.stdout[-4000:])
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "0 failure(s)" in r.stdout
