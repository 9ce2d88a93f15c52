"""GPU: the reference's own unit tests (heston.rs, bates.rs, batch.rs,
calibration.rs), ported to C++ against the C++ API mirror, run on the GPU."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_reference_unit_tests_through_cpp_mirror(ope):
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "cpp")])
    p = subprocess.run([os.path.join(HERE, "cpp", "reference_suite")], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "FAIL" not in p.stdout and p.stdout.count("PASS") >= 20, p.stdout
