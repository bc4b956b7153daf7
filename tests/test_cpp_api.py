"""The C++ host API (include/xatu_bse.hpp over the C ABI) from a compiled C++ program shaped like the
reference's main/minimal_example.cpp:13-19: read a .model, build the exciton, initializeHamiltonian,
BShamiltonian, diagonalize.  The program is built with g++ against the in-tree library.  On the CPU it
checks that the program compiles and that its .model reader agrees with the Python reader; on the GPU it
runs MoS2 with exchange and Q != 0 and meets the reference's MoS2_exchange golden (tests.cpp:704-737)
through both the FP64 dense path and the mixed Davidson path."""
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import detect_degeneracies
from tests.helpers import MODELS, goldens, model_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "xatu_b200", "_lib")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from xatu_b200 import _lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.skip("engine library not built")
    exe = str(tmp_path_factory.mktemp("cpp") / "minimal_example")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "minimal_example.cpp"), "-L" + LIBDIR, "-lxatu_bse",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("model", ["hBN.model", "MoS2.model", "hBN_spinful.model"])
def test_cpp_model_reader_matches_python(program, model):
    r = subprocess.run([program, "parse", os.path.join(MODELS, model)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    f = r.stdout.split()
    vals = dict(zip(f[0::2], f[1::2]))
    si = model_config(model).systemInfo
    assert int(vals["ndim"]) == si.ndim
    assert int(vals["natoms"]) == si.motif.shape[0]
    assert int(vals["species"]) == len(si.norbitals)
    assert int(vals["norb"]) == si.hamiltonian.shape[1]
    assert int(vals["ncells"]) == si.hamiltonian.shape[0]
    assert int(vals["filling"]) == int(si.filling)
    assert float(vals["sum|H|"]) == pytest.approx(float(np.abs(si.hamiltonian).sum()), rel=1e-12)


def test_cpp_reader_rejects_missing_file(program):
    r = subprocess.run([program, "parse", os.path.join(MODELS, "missing.model")], capture_output=True, text=True)
    assert r.returncode == 1 and "does not exist" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision,method", [("fp64", "diag"), ("mixed", "davidson")])
def test_cpp_minimal_example_mos2_exchange_golden(program, precision, method):
    case = next(c for c in goldens()["cases"] if c["name"] == "MoS2_exchange")
    Q = case["extra"]["Q"]
    n = case["nstates"]
    eps_m, eps_s, r0 = case["params"]
    args = [program, os.path.join(MODELS, case["model"]), str(case["ncell"]), str(case["nbands"]), str(eps_m),
            str(eps_s), str(r0), str(Q[0]), str(Q[1]), str(Q[2]), "1", precision, method,
            str(n if method == "diag" else n + 2)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    energies = np.array([float(line.split()[2]) for line in r.stdout.splitlines() if line.startswith("E ")])
    pairs = detect_degeneracies(energies, n, 6 if precision == "fp64" else 5)
    for (e, d), (ee, dd) in zip(pairs, case["expected"]):
        assert e == pytest.approx(ee, abs=case["tol"])
        assert d == dd
