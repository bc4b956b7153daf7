"""Input readers against the reference's parsing goldens (tests.cpp:19-61, :125-148)."""
import os

import numpy as np
import pytest

from oracle.oracle import array2hash
from tests.helpers import GOLDEN, MODELS, goldens
from xatu_b200.config import ExcitonConfiguration, SystemConfiguration


def test_model_parsing_hashes():
    g = goldens()["hashes"]["model_parsing"]
    cfg = SystemConfiguration(os.path.join(MODELS, g["file"]))
    si = cfg.systemInfo
    assert si.ndim == g["ndim"]
    assert si.filling == g["filling"]
    assert list(si.norbitals) == g["orbitals"]
    # rows are Armadillo subview_rows in the reference test: hashed with aliasing
    for i, h in enumerate(g["bravais_hash"]):
        assert array2hash(si.bravaisLattice[i][None, :], subview=True) == pytest.approx(h, abs=g["tol"])
    for i, h in enumerate(g["motif_hash"]):
        assert array2hash(si.motif[i][None, :], subview=True) == pytest.approx(h, abs=g["tol"])
    for i, h in enumerate(g["bravais_vectors_hash"]):
        assert array2hash(si.bravaisVectors[i][None, :], subview=True) == pytest.approx(h, abs=g["tol"])
    for i, h in enumerate(g["hamiltonian_hash"]):
        assert array2hash(si.hamiltonian[i]) == pytest.approx(h, abs=g["tol"])


def test_exciton_file_parsing():
    g = goldens()["hashes"]["exciton_parsing"]
    cfg = ExcitonConfiguration(os.path.join(GOLDEN, g["file"]))
    info = cfg.excitonInfo
    assert info.label.strip() == g["label"]
    assert info.ncell == g["ncell"]
    assert info.nbands == g["nbands"]
    assert list(info.eps) == g["dielectric"]
    assert array2hash(info.Q[None, :]) == 0


def test_spinful_and_mos2_models_parse():
    s = SystemConfiguration(os.path.join(MODELS, "hBN_spinful.model")).systemInfo
    assert s.hamiltonian.shape == (5, 4, 4)
    m = SystemConfiguration(os.path.join(MODELS, "MoS2.model")).systemInfo
    assert list(m.norbitals) == [10, 6]
    assert m.hamiltonian.shape[1:] == (22, 22)
    assert m.hamiltonian.shape[0] == m.bravaisVectors.shape[0]
    # Hermiticity of the Bloch sum needs H(-R) = H(R)^dagger for every stored pair
    H = m.hamiltonian
    R = m.bravaisVectors
    for i in range(R.shape[0]):
        j = int(np.argmin(np.linalg.norm(R + R[i], axis=1)))
        assert np.allclose(H[j], H[i].conj().T, atol=1e-9)


def test_parser_errors(tmp_path):
    bad = tmp_path / "bad.model"
    bad.write_text("# dimension\n2\n# norbitals\n1 1\n# filling\n1\n")
    with pytest.raises(ValueError):
        SystemConfiguration(str(bad))
    with pytest.raises(ValueError):
        SystemConfiguration(str(tmp_path / "missing.model"))
    ex = tmp_path / "ex.txt"
    ex.write_text("# ncells\n10\n# bands\n1\n# dielectric\n1 1 10\n# exchange\nmaybe\n")
    with pytest.raises(ValueError):
        ExcitonConfiguration(str(ex))
