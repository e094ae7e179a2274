"""The C++ mirror of the reference API (linear-massiv_b200/host/massiv.hpp),
compiled against the C ABI and run on the GPU: the reference's known-answer
cases through compile-time-dimensioned Matrix<M, N> / Vector<N>."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_mirror_known_answers(tmp_path):
    pkg = os.path.join(ROOT, "linear-massiv_b200")
    exe = str(tmp_path / "massiv_example")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(pkg, "host"),
                    os.path.join(pkg, "host", "example.cpp"), "-L" + pkg, "-llm_b200", "-Wl,-rpath," + pkg,
                    "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 failure(s)" in out.stdout
