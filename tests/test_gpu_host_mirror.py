"""The C++ mirror of the reference API (linear-massiv_b200/host/massiv.hpp),
compiled against the C ABI and run on the GPU: the reference's known-answer
cases through compile-time-dimensioned Matrix<M, N> / Vector<N>, and systems
whose size is known only at run time (SomeMatrix, someMatrix, reifyDim)
against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, philox
from helpers import backward_error, gen_spd, gen_uniform, rel_forward

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    pkg = os.path.join(ROOT, "linear-massiv_b200")
    path = str(tmp_path_factory.mktemp("mirror") / "massiv_example")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(pkg, "host"),
                    os.path.join(pkg, "host", "example.cpp"), "-L" + pkg, "-llm_b200", "-Wl,-rpath," + pkg,
                    "-o", path], check=True)
    return path


@pytest.mark.parametrize("n,kind", [(3, 0), (64, 0), (300, 1), (777, 0), (1500, 1), (2049, 0)])
def test_cpp_mirror_runtime_sizes_vs_oracle(exe, tmp_path, n, kind):
    """A system whose size the program learns from its input: sizes among the
    reifyDim candidates (3, 64, 300) run the typed API, the others SomeMatrix."""
    g = philox(35000 + n)
    A = gen_spd(g, n) if kind == 1 else gen_uniform(g, n)
    b = g.uniform(-1, 1, n)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(np.array([kind, n], dtype=np.int32).tobytes() + A.tobytes() + b.tobytes())
    out = subprocess.run([exe, "solve", str(fin), str(fout)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert ("typed API" in out.stdout) == (n in (3, 64, 300))
    x = np.fromfile(fout, dtype=np.float64)
    xo = (O.lu_solve_p(A, b) if kind == 0 else O.chol_solve_p(A, b))[0]
    assert backward_error(A, x, b) <= 1e-15 * n
    bar = 1e-12 if kind == 1 else max(1e-12, 32 * np.linalg.cond(A) * EPS)
    assert rel_forward(x, xo) <= bar


def test_cpp_mirror_known_answers(exe):
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 failure(s)" in out.stdout
