"""The CPU oracle against the reference's own golden values (test/tests.cpp).

This pins the oracle: its restatement of the build (C) and solve (LAPACK
zheevd via numpy) reproduces every golden exciton energy of the BSE hot path
and the k-space wavefunction hashes."""
import numpy as np
import pytest

from oracle.oracle import array2hash, detect_degeneracies
from tests.helpers import case_kwargs, goldens, model_config, oracle_exciton

CASES = goldens()["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_energies(case):
    cfg = model_config(case["model"])
    ex = oracle_exciton(cfg, case["ncell"], case["nbands"], case["params"], **case_kwargs(case))
    ex.bs_hamiltonian()
    method = case["extra"].get("method", "diag")
    n = case["nstates"]
    if method == "davidson":
        w, _ = ex.diagonalize("davidson", n)
    else:
        w, _ = ex.diagonalize("diag")
    pairs = detect_degeneracies(w, n, 6)
    for (e, d), (ee, dd) in zip(pairs, case["expected"]):
        assert e == pytest.approx(ee, abs=case["tol"])
        assert d == dd


@pytest.mark.parametrize("key", ["hBN_kwf", "MoS2_kwf"])
def test_oracle_kwf_hash(key):
    g = goldens()["hashes"][key]
    cfg = model_config(g["model"])
    ex = oracle_exciton(cfg, g["ncell"], g["nbands"], g["params"])
    ex.bs_hamiltonian()
    w, v = ex.diagonalize("diag")
    ncv = len(ex.valence) * len(ex.conduction)
    nk = ex.kpoints.shape[0]
    dk = np.linalg.norm(ex.kpoints[1] - ex.kpoints[0])
    kwf = np.zeros(nk, dtype=complex)
    for s in range(g["nstates"]):
        c = v[:, s]
        kwf += (np.abs(c.reshape(nk, ncv)) ** 2).sum(axis=1) / dk
    assert array2hash(kwf) == pytest.approx(g["hash"], abs=g["tol"])


@pytest.mark.parametrize("model,ncell,nbands,params,golden", [
    ("hBN.model", 20, 1, [1, 1, 10], 47.4140063784),          # tests.cpp:371-399
    ("MoS2.model", 12, 2, [1., 4., 13.55], 37.2792093358),    # tests.cpp:776-804
])
def test_oracle_oscillator_strength_sum(model, ncell, nbands, params, golden):
    from oracle.oracle import exciton_oscillator_strength
    ex = oracle_exciton(model_config(model), ncell, nbands, params)
    ex.bs_hamiltonian()
    w, v = ex.diagonalize("diag")
    vx = exciton_oscillator_strength(ex, v)
    assert float(np.sum(np.abs(vx) ** 2)) == pytest.approx(golden, abs=1e-7)


def test_oracle_matrix_is_hermitian_and_diag_real():
    cfg = model_config("MoS2.model")
    ex = oracle_exciton(cfg, 6, 2, [1., 4., 13.55], Q=(0, 0.1, 0), exchange=True)
    H = ex.bs_hamiltonian()
    assert np.array_equal(H, H.conj().T)
    assert np.all(np.diag(H).imag == 0)


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's inputs is visible in the energies (the check has teeth)."""
    cfg = model_config("hBN.model")
    ex = oracle_exciton(cfg, 8, 1, [1, 1, 10])
    H0 = ex.bs_hamiltonian().copy()
    ex.ft_stack = ex.ft_stack * 1.01
    H1 = ex.bs_hamiltonian()
    assert np.abs(np.linalg.eigvalsh(H0)[0] - np.linalg.eigvalsh(H1)[0]) > 1e-4
