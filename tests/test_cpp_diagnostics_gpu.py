"""Build and run tests/cpp/test_diagnostics.cpp: the C++ drop-ins of
include/granite_b200_diagnostics.hpp (MatterSources, Psi4Extractor,
ApparentHorizonFinder) linked to libgranite_ccz4.so. The compile step runs
everywhere; the run needs the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_binary(tmp_path):
    from granite_b200 import build
    lib = build.build()
    exe = tmp_path / "test_diagnostics"
    subprocess.run([CXX, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "test_diagnostics.cpp"), "-o", str(exe),
                    lib, f"-Wl,-rpath,{os.path.dirname(lib)}"], check=True)
    return exe


def test_diagnostics_compile(tmp_path):
    assert build_binary(tmp_path).exists()


@pytest.mark.gpu
def test_diagnostics_dropins(tmp_path):
    exe = build_binary(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout
