"""CPU restatement of the exciton post-processing -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy and FP64, the observables and writers of Xatu v1.3.1 that
consume the eigen-pairs of the BSE:

  * Result.tpp:25-40     kineticEnergy          (band part of the exciton energy)
  * Result.tpp:101-128   ftExcitonEnvelope      (Fourier transform of |A(k)|^2)
  * Result.tpp:160-179   writeReciprocalAmplitude (per-k weights / |k1 - k0|)
  * Result.tpp:478-484   findExcitonPeak, :76-89 determineGap
  * ResultTB.cpp:21-98   spinX                  (Sz of electron and hole)
  * ResultTB.cpp:310-357 realSpaceWavefunction, :470-481 addExponential
  * skubo_w.f90:2-173    skubo_w (single-particle Kubo and exciton absorption),
    :630-681 get_kubo_intens, :684-720 broad_vector

It is the checker for the device post-processing entry points; only the test
suite imports it.  Pinned by tests/test_oracle_postproc.py against the
reference's golden real-space and k-space wavefunction hashes and spin values
(test/tests.cpp:281-369, :402-462).
"""
from __future__ import annotations

import numpy as np

from .oracle import BOHR, HARTREE, exciton_oscillator_strength, vme_single_particle

PI = np.arccos(-1.0)


def _orbital_range(system, atom: int):
    off = int(system.orb_offset[atom])
    return off, int(system.orb_offset[atom + 1]) - off


def add_exponential(ex, coefs: np.ndarray, cell) -> np.ndarray:
    """ResultTB::addExponential (ResultTB.cpp:470-481): coefs(k, c, v) * exp(i k . cell)."""
    product = ex.kpoints @ np.asarray(cell, dtype=np.float64)
    nbc = len(ex.valence) * len(ex.conduction)
    return coefs * np.repeat(np.exp(1j * product), nbc)


def real_space_wavefunction(ex, coefs: np.ndarray, electron_index: int, hole_index: int, e_cell, h_cell) -> float:
    """ResultTB::realSpaceWavefunction (ResultTB.cpp:310-357): sum over the orbitals alpha of the
    electron atom and beta of the hole atom of |sum_{k,c,v} C^Q_{k,c}[alpha] conj(C_{k,v}[beta])
    A(k,c,v) e^{i k.(Re - Rh)}|^2 (arma::dot: no conjugation of either operand)."""
    s = ex.system
    nv, nc = len(ex.valence), len(ex.conduction)
    nk = ex.kpoints.shape[0]
    e_off, e_orb = _orbital_range(s, electron_index)
    h_off, h_orb = _orbital_range(s, hole_index)
    x = add_exponential(ex, np.asarray(coefs, dtype=np.complex128),
                        np.asarray(e_cell, dtype=np.float64) - np.asarray(h_cell, dtype=np.float64))
    total = 0.0
    for alpha in range(e_orb):
        for beta in range(h_orb):
            c_flat = ex.eigvecQ[:, nv:nv + nc, e_off + alpha].reshape(-1)     # index k*nc + c
            c_ext = np.repeat(c_flat, nv)                                      # kron(cFlat, ones(nv))
            v = ex.eigvec[:, :nv, h_off + beta]                                # (nk, nv)
            v_ext = np.tile(v, (1, nc)).reshape(nk * nc * nv)                  # per k: kron(ones(nc), v_k)
            amp = np.dot(c_ext * np.conj(v_ext), x)
            total += float(amp.real ** 2 + amp.imag ** 2)
    return total


def realspace_amplitudes(ex, coefs: np.ndarray, hole_index: int, hole_cell, cells: np.ndarray) -> np.ndarray:
    """The loop of writeRealspaceAmplitude (ResultTB.cpp:370-408): values[cell][atom]."""
    na = ex.system.natoms
    out = np.zeros((cells.shape[0], na))
    for ci in range(cells.shape[0]):
        for atom in range(na):
            out[ci, atom] = real_space_wavefunction(ex, coefs, atom, hole_index, cells[ci], hole_cell)
    return out


def kinetic_energy(ex, coefs: np.ndarray) -> float:
    """Result::kineticEnergy (Result.tpp:25-40): cdot(A, HK % A), HK = E^Q_c(k) - E_v(k) (no scissor)."""
    nv, nc = len(ex.valence), len(ex.conduction)
    nk = ex.kpoints.shape[0]
    hk = (ex.eigvalQ[:, nv:nv + nc][:, :, None] - ex.eigval[:, :nv][:, None, :]).reshape(nk * nc * nv)
    a = np.asarray(coefs, dtype=np.complex128)
    return float(np.vdot(a, hk * a).real)


def reciprocal_weights(ex, coefs: np.ndarray) -> np.ndarray:
    """sum_{c,v} |A(k,c,v)|^2 per k (the numerator of writeReciprocalAmplitude, Result.tpp:160-179)."""
    nbc = len(ex.valence) * len(ex.conduction)
    a = np.asarray(coefs, dtype=np.complex128).reshape(-1, nbc)
    return (np.abs(a) * np.abs(a)).sum(axis=1)


def reciprocal_amplitude(ex, coefs: np.ndarray) -> np.ndarray:
    """writeReciprocalAmplitude's per-k value (Result.tpp:167-173): weights / |k1 - k0|."""
    return reciprocal_weights(ex, coefs) / np.linalg.norm(ex.kpoints[1] - ex.kpoints[0])


def ft_exciton_envelope(ex, coefs: np.ndarray, electron_position, hole_position) -> float:
    """Result::ftExcitonEnvelope (Result.tpp:101-128): Re sum_k |A_k|^2 exp(-i k.(re - rh))."""
    w = reciprocal_weights(ex, coefs)
    d = np.asarray(electron_position, dtype=np.float64) - np.asarray(hole_position, dtype=np.float64)
    return float(np.real(np.sum(w * np.exp(-1j * (ex.kpoints @ d)))))


def find_exciton_peak(ex, coefs: np.ndarray) -> int:
    """Result::findExcitonPeak (Result.tpp:478-484): k index of the largest |coefficient|."""
    nbc = len(ex.valence) * len(ex.conduction)
    return int(np.argmax(np.abs(np.asarray(coefs)))) // nbc


def determine_gap(ex, coefs0: np.ndarray) -> float:
    """Result::determineGap (Result.tpp:76-89) at the peak of the given (ground) state."""
    k = find_exciton_peak(ex, coefs0)
    nv = len(ex.valence)
    iv = int(np.argmax(ex.valence))           # bandToIndex[max(valenceBands)]
    ic = nv + int(np.argmin(ex.conduction))   # bandToIndex[min(conductionBands)]
    return float(ex.eigval[k, ic] - ex.eigval[k, iv])


def spin_vector(system) -> np.ndarray:
    """Sz of every orbital (ResultTB.cpp:30-37): +1/2, -1/2 alternating within each atom."""
    out = np.zeros(system.basisdim)
    for atom in range(system.natoms):
        off, n = _orbital_range(system, atom)
        if n % 2:
            raise ValueError("spinX needs an even number of orbitals on every atom")
        out[off:off + n] = np.kron(np.ones(n // 2), [0.5, -0.5])
    return out


def spin_x(ex, coefs: np.ndarray) -> np.ndarray:
    """ResultTB::spinX (ResultTB.cpp:21-98): [total, hole, electron] with the per-k blocks
    kron(I_nc, S_hole) and kron(S_electron, I_nv) of the reference."""
    s = ex.system
    sv = spin_vector(s)
    nv, nc = len(ex.valence), len(ex.conduction)
    nk = ex.kpoints.shape[0]
    npairs = nv * nc
    a = np.asarray(coefs, dtype=np.complex128)
    hole = 0j
    elec = 0j
    for k in range(nk):
        C = ex.eigvec[k]       # (nb, norb)
        CQ = ex.eigvecQ[k]
        sh = np.zeros((nv, nv), dtype=np.complex128)
        for i in range(nv):
            for j in range(nv):
                sh[i, j] = np.vdot(C[j], C[i] * sv)
        se = np.zeros((nc, nc), dtype=np.complex128)
        for i in range(nc):
            for j in range(nc):
                se[i, j] = np.vdot(CQ[nv + i], CQ[nv + j] * sv)
        blk = a[k * npairs:(k + 1) * npairs]
        hole += np.vdot(blk, np.kron(np.eye(nc), sh) @ blk)
        elec += np.vdot(blk, np.kron(se, np.eye(nv)) @ blk)
    hole = -hole
    return np.array([np.real(hole + elec), hole, elec], dtype=np.complex128)


# ----------------------------------------------------------------------------- absorption


def cell_area_bohr(system) -> float:
    """vcell of skubo_w (skubo_w.f90:69-71): |a1 x a2| in bohr^2 with the lattice padded to 3 x 3."""
    R = np.zeros((3, 3))
    R[:system.bravais.shape[0]] = system.bravais
    R = R / BOHR
    return float(np.linalg.norm(np.cross(R[0], R[1])))


def frequencies(w0: float, wrange: float, nw: int) -> np.ndarray:
    """wp(i) of skubo_w (skubo_w.f90:88-90), Hartree."""
    return np.array([(w0 + wrange / nw * i) / HARTREE for i in range(nw)])


def broad_vector(kind: str, wn: np.ndarray, fn: np.ndarray, wp: np.ndarray, eta: float) -> np.ndarray:
    """broad_vector (skubo_w.f90:684-720): sum_n Re(fn) * broadening(wp - wn); an unknown kind keeps 1."""
    out = np.zeros(len(wp))
    for i, w in enumerate(wp):
        acc = 0.0
        for e, f in zip(wn, np.real(fn)):
            r = 1.0
            if kind == "lorentzian":
                r = 1.0 / PI * np.imag(1.0 / (w - e - 1j * eta))
            if kind == "gaussian":
                r = 1.0 / eta * 1.0 / np.sqrt(2.0 * PI) * np.exp(-0.5 / eta ** 2 * (w - e) ** 2)
            if kind == "exponential":
                r = 0.5 / eta * np.exp(-abs(w - e) / eta)
            acc += f * r
        out[i] = acc
    return out


def kubo_single_particle(ex, w0: float, wrange: float, nw: int, eta_ev: float) -> np.ndarray:
    """Single-particle Kubo conductivity of skubo_w (skubo_w.f90:103-110) with get_kubo_intens
    (skubo_w.f90:630-681): sigma_sp[w][3][3], complex (the file holds -Re)."""
    s = ex.system
    nv = len(ex.valence)
    nb = len(ex.band_list)
    nk = ex.kpoints.shape[0]
    vcell = cell_area_bohr(s)
    wp = frequencies(w0, wrange, nw)
    eta = eta_ev / HARTREE
    sigma = np.zeros((nw, 3, 3), dtype=np.complex128)
    pref = PI / (float(nk) * vcell)
    for ik in range(nk):
        e = ex.eigval[ik] / HARTREE
        vme = vme_single_particle(s, ex.kpoints[ik] * BOHR, ex.eigvec[ik].T, e)
        for nn in range(nb):
            fnn = 1.0 if nn < nv else 0.0
            for nnp in range(nb):
                fnnp = 1.0 if nnp < nv else 0.0
                if abs(fnn - fnnp) < 0.1:
                    continue   # factor1 = 0
                factor1 = (fnn - fnnp) / (e[nn] - e[nnp])
                delta = 1.0 / eta * 1.0 / np.sqrt(2.0 * PI) * np.exp(-0.5 / eta ** 2 * (wp - e[nn] + e[nnp]) ** 2)
                sk = vme[:, nn, nnp][:, None] * vme[:, nnp, nn][None, :]
                sigma += (pref * factor1) * sk[None, :, :] * delta[:, None, None]
    return sigma


def exciton_absorption(ex, eigval: np.ndarray, eigvec: np.ndarray, w0: float, wrange: float, nw: int,
                       eta_ev: float, kind: str):
    """Exciton part of skubo_w (skubo_w.f90:113-130): (sigma_ex[w][3][3] real, vme_ex[3][ns])."""
    s = ex.system
    nk = ex.kpoints.shape[0]
    vcell = cell_area_bohr(s)
    wp = frequencies(w0, wrange, nw)
    eta = eta_ev / HARTREE
    e_ex = np.asarray(eigval, dtype=np.float64) / HARTREE
    vme_ex = exciton_oscillator_strength(ex, np.asarray(eigvec, dtype=np.complex128))
    sigma = np.zeros((nw, 3, 3))
    pref = PI / (float(nk) * vcell)
    for a in range(2):
        for b in range(2):
            fn = pref * np.conj(vme_ex[a]) * vme_ex[b] / e_ex
            sigma[:, a, b] = broad_vector(kind, e_ex, fn, wp, eta)
    return sigma, vme_ex
