"""The post-processing restatement (oracle/postproc.py) against the reference's own goldens, and the host
helpers of xatu_b200.result that need no GPU.

Pins: the real-space wavefunction hash of hBN (tests.cpp:323-369) and the spin values of spinful hBN
(tests.cpp:432-462); the k-space hashes are pinned in test_oracle_golden.py."""
import numpy as np
import pytest

from oracle.oracle import array2hash, generate_combinations, truncate_supercell
from oracle.postproc import (broad_vector, exciton_absorption, find_exciton_peak, ft_exciton_envelope,
                             kinetic_energy, real_space_wavefunction, realspace_amplitudes, reciprocal_weights,
                             spin_x)
from tests.helpers import goldens, model_config, oracle_exciton
from xatu_b200.result import generate_combinations as gen_comb_product
from xatu_b200.result import read_kubo_parameters


def _solved(g):
    ex = oracle_exciton(model_config(g["model"]), g["ncell"], g["nbands"], g["params"])
    ex.bs_hamiltonian()
    w, v = ex.diagonalize("diag")
    return ex, w, v


def _rswf(ex, v, g, hole_index=None):
    s = ex.system
    cells = truncate_supercell(s.bravais, s.ndim, g["ncell"], np.linalg.norm(s.bravais[0]) * g["radius_cells"])
    hole = g["hole_index"] if hole_index is None else hole_index
    rs = np.zeros(cells.shape[0] * s.natoms)
    for n in range(g["nstates"]):
        rs += realspace_amplitudes(ex, v[:, n], hole, np.asarray(g["hole_cell"], float), cells).reshape(-1)
    return rs


def test_oracle_realspace_hash():
    g = goldens()["hashes"]["hBN_rswf"]
    ex, w, v = _solved(g)
    assert array2hash(_rswf(ex, v, g)) == pytest.approx(g["hash"], abs=g["tol"])


def test_oracle_realspace_hash_detects_wrong_hole():
    """A planted mistake in the oracle's inputs (hole on the other atom) moves the hash off the golden."""
    g = goldens()["hashes"]["hBN_rswf"]
    ex, w, v = _solved(g)
    assert abs(array2hash(_rswf(ex, v, g, hole_index=0)) - g["hash"]) > 1e-3


def test_oracle_spin_golden():
    g = goldens()["hashes"]["hBN_spin"]
    ex, w, v = _solved(g)
    for i in range(g["nstates"]):
        sp = spin_x(ex, v[:, i])
        assert sp[0].real == pytest.approx(g["total"][i], abs=g["tol"])
        assert abs(sp[1]) == pytest.approx(g["abs_parts"], abs=g["tol"])
        assert abs(sp[2]) == pytest.approx(g["abs_parts"], abs=g["tol"])


def test_oracle_spin_needs_even_orbitals():
    g = goldens()["hashes"]["hBN_rswf"]     # spinless hBN: one orbital per atom
    ex, w, v = _solved(g)
    with pytest.raises(ValueError):
        spin_x(ex, v[:, 0])


def test_oracle_observables_consistent():
    """Identities between the restated observables: the envelope transform at zero separation is the norm,
    the kinetic energy lies within the band-gap range, the single-cell amplitude matches the loop."""
    g = goldens()["hashes"]["hBN_rswf"]
    ex, w, v = _solved(g)
    x = v[:, 0]
    assert ft_exciton_envelope(ex, x, np.zeros(3), np.zeros(3)) == pytest.approx(1.0, abs=1e-12)
    assert reciprocal_weights(ex, x).sum() == pytest.approx(1.0, abs=1e-12)
    nv = len(ex.valence)
    gaps = ex.eigvalQ[:, nv:] .min(axis=1) - ex.eigval[:, :nv].max(axis=1)
    kin = kinetic_energy(ex, x)
    assert gaps.min() - 1e-12 <= kin <= (ex.eigvalQ[:, nv:].max() - ex.eigval[:, :nv].min()) + 1e-12
    k = find_exciton_peak(ex, x)
    assert 0 <= k < ex.kpoints.shape[0]
    a = real_space_wavefunction(ex, x, 0, 1, np.zeros(3), np.zeros(3))
    b = realspace_amplitudes(ex, x, 1, np.zeros(3), np.zeros((1, 3)))[0, 0]
    assert a == b


def test_oracle_absorption_sum_rule():
    """Gaussian-broadened exciton conductivity integrates to the summed oscillator weights when the window
    covers every peak (broad_vector is a sum of unit-area kernels)."""
    g = goldens()["hashes"]["hBN_rswf"]
    ex, w, v = _solved(g)
    ns = 6
    sig, vme = exciton_absorption(ex, w[:ns], v[:, :ns], 0.0, 12.0, 3000, 0.1, "gaussian")
    from oracle.oracle import HARTREE
    from oracle.postproc import PI, cell_area_bohr
    pref = PI / (ex.kpoints.shape[0] * cell_area_bohr(ex.system))
    weights = (pref * np.conj(vme[0]) * vme[0] / (w[:ns] / HARTREE)).real
    dw = 12.0 / 3000 / HARTREE
    assert sig[:, 0, 0].sum() * dw == pytest.approx(weights.sum(), rel=1e-6)
    assert np.all(sig[:, 2, :] == 0) and np.all(sig[:, :, 2] == 0)


def test_broad_vector_kinds():
    wn = np.array([0.1, 0.2])
    fn = np.array([1.0 + 2j, 3.0])
    wp = np.linspace(0, 0.3, 7)
    eta = 0.01
    lor = broad_vector("lorentzian", wn, fn, wp, eta)
    ref = sum(f * eta / np.pi / ((wp - e) ** 2 + eta ** 2) for e, f in zip(wn, [1.0, 3.0]))
    assert np.allclose(lor, ref, rtol=1e-13, atol=0)
    # an unknown kind keeps weight 1 (skubo_w.f90:703)
    assert np.allclose(broad_vector("none", wn, fn, wp, eta), 4.0)


def test_generate_combinations_matches_oracle():
    for nv, nd in ((3, 1), (3, 2), (3, 3), (4, 2)):
        assert np.array_equal(gen_comb_product(nv, nd, True), generate_combinations(nv, nd, True))
        assert np.array_equal(gen_comb_product(nv, nd, False), generate_combinations(nv, nd, False))


def test_read_kubo_parameters(tmp_path):
    """The kubo_w.in layout of the reference: comment / value pairs, Fortran 'd' exponent, two file names."""
    p = tmp_path / "kubo_w.in"
    p.write_text("#initial frequency (eV)\n1\n#frequency range (eV)\n6\n#number of frequency points (integer)\n"
                 "400\n#broadening parameter (eV)\n0.08d0\n#type of broadening\nlorentzian\n#output kubo name files\n"
                 "hBN_sp.dat\nhBN_ex.dat")
    prm = read_kubo_parameters(str(p))
    assert prm == {"w0": 1.0, "wrange": 6.0, "nw": 400, "eta": 0.08, "broadening": "lorentzian",
                   "file_sp": "hBN_sp.dat", "file_ex": "hBN_ex.dat"}
    p.write_text("#x\n1\n")
    with pytest.raises(ValueError):
        read_kubo_parameters(str(p))
