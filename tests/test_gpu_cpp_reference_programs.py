"""The reference's test programs (test/test1.cu, test/binTest_Broadphase.cu,
test/nSquared_Broadphase.cu) plus a full GenerateAABB -> Broadphase ->
Narrowphase step, written against include/collide_b200.hpp exactly as a
reference caller writes them (tests/cpp/reference_tests.cu)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "build", "reference_tests")


@pytest.mark.parametrize("which", ["test1", "bintest", "nsquared", "pipeline"])
def test_reference_program(cb, which):
    if not os.path.exists(EXE):
        subprocess.run(["make", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    r = subprocess.run([EXE, which], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "TEST PASSED" in r.stdout and "TEST FAILED" not in r.stdout, r.stdout + r.stderr
