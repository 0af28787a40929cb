"""The integration code against the reference itself: tests/cpp/reference_integration.cpp
compiled against the reference's headers (-Wall -Wextra -Werror), linked with its
grid.cpp and amr.cpp and with libgranite_ccz4.so (the `integration` target of
oracle/Makefile). Its main() builds a reference AMRHierarchy from a tracking
sphere and checks that the block descriptors the wrappers pass to the C ABI
reproduce every GridBlock's geometry; without a GPU the library must answer
GRANITE_ERR_NO_DEVICE. Skipped where the reference tree is absent."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "reference_integration")


def test_integration_code_builds_against_the_reference_and_runs():
    from granite_b200 import build
    build.build()
    mk = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "integration"], capture_output=True,
                        text=True, timeout=600)
    assert mk.returncode == 0, mk.stdout[-2000:] + mk.stderr[-2000:]
    if not os.path.exists(EXE):
        pytest.skip("reference tree not present: integration build skipped")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "OK (0 failures)" in r.stdout
    assert "3 blocks on 3 levels mirrored" in r.stdout
