"""Seeded synthetic tight-binding models for the benchmark workloads.

``synthetic_hexagonal`` builds the 3-atom hexagonal model of the headline
workload: species orbitals 8 + 7 + 7 = 22, Hermitian complex hoppings drawn
from N(0, sigma) to the first and second neighbour cells, on-site energies
U(-2, 2) eV on a Hermitian R = 0 block.  H(-R) = H(R)^dagger is stored
explicitly (the Bloch sum of SystemTB::hamiltonian does not hermitise full
matrices, SystemTB.cpp:60-75).  The returned object quacks like a
SystemConfiguration (``.systemInfo``) so it feeds ExcitonTB directly.

``random_honeycomb`` draws the small 2-12 orbital honeycomb models of the
batched workload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .config import SystemInfo


@dataclass
class SyntheticConfiguration:
    systemInfo: SystemInfo
    seed: int
    description: str


def _hex_cells(a1: np.ndarray, a2: np.ndarray, shells: int):
    """R = 0 followed by +/- pairs of the first (and second) neighbour cells."""
    first = [(1, 0), (0, 1), (1, -1)]
    second = [(1, 1), (2, -1), (-1, 2)]
    pos = first + (second if shells >= 2 else [])
    cells = [np.zeros(3)]
    for (m, n) in pos:
        cells.append(m * a1 + n * a2)
    for (m, n) in pos:
        cells.append(-(m * a1 + n * a2))
    return np.array(cells), len(pos)


def _herm_random(rng, n, sigma):
    re = rng.normal(0.0, sigma / math.sqrt(2), size=(n, n))
    im = rng.normal(0.0, sigma / math.sqrt(2), size=(n, n))
    return re + 1j * im


def synthetic_hexagonal(seed: int = 1234, orbitals=(8, 7, 7), a: float = 3.0, sigma: float = 0.5,
                        onsite: float = 2.0, shells: int = 2, filling: int | None = None,
                        overlap: float = 0.0) -> SyntheticConfiguration:
    """``overlap`` > 0 adds non-orthogonal-basis overlap matrices S(R): identity plus
    Hermitian random terms of that size on R = 0 and on the neighbour cells."""
    rng = np.random.default_rng(seed)
    a1 = np.array([a, 0.0, 0.0])
    a2 = np.array([a / 2, a * math.sqrt(3) / 2, 0.0])
    frac = [(0.0, 0.0), (1 / 3, 1 / 3), (2 / 3, 2 / 3)]
    species = [0, 1, 1] if len(orbitals) == 3 and orbitals[1] == orbitals[2] else list(range(len(orbitals)))
    norb_species = sorted(set(species))
    norbitals = np.array([orbitals[species.index(s)] for s in norb_species], dtype=np.int64)
    motif = np.array([[*(f0 * a1 + f1 * a2)[:3], float(sp)] for (f0, f1), sp in zip(frac, species)])
    norb = int(sum(orbitals))
    cells, npos = _hex_cells(a1, a2, shells)
    H = np.zeros((cells.shape[0], norb, norb), dtype=np.complex128)
    h0 = _herm_random(rng, norb, sigma)
    h0 = 0.5 * (h0 + h0.conj().T)
    np.fill_diagonal(h0, rng.uniform(-onsite, onsite, size=norb))
    H[0] = h0
    for p in range(npos):
        hr = _herm_random(rng, norb, sigma)
        H[1 + p] = hr
        H[1 + npos + p] = hr.conj().T
    info = SystemInfo()
    if overlap > 0:
        S = np.zeros_like(H)
        s0 = _herm_random(rng, norb, overlap)
        S[0] = np.eye(norb) + 0.5 * (s0 + s0.conj().T)
        for p in range(npos):
            sr = _herm_random(rng, norb, overlap * 0.5)
            S[1 + p] = sr
            S[1 + npos + p] = sr.conj().T
        info.overlap = S
    info.ndim = 2
    info.filling = float(filling if filling is not None else norb // 2)
    info.bravaisLattice = np.array([a1, a2])
    info.motif = motif
    info.hamiltonian = H
    info.bravaisVectors = cells
    info.norbitals = norbitals
    return SyntheticConfiguration(info, seed, f"synthetic hexagonal {'+'.join(map(str, orbitals))} orbitals, "
                                              f"sigma={sigma} eV, seed={seed}")


def random_honeycomb(seed: int, norb_total: int) -> SyntheticConfiguration:
    """Two-atom honeycomb with norb_total = 2..12 orbitals split over the two atoms."""
    rng = np.random.default_rng(seed)
    a = 2.5
    a1 = np.array([a * math.sqrt(3) / 2, a / 2, 0.0])
    a2 = np.array([a * math.sqrt(3) / 2, -a / 2, 0.0])
    n0 = max(1, norb_total // 2)
    n1 = max(1, norb_total - n0)
    motif = np.array([[0.0, 0.0, 0.0, 0.0], [a / math.sqrt(3), 0.0, 0.0, 1.0]])
    norb = n0 + n1
    cells, npos = _hex_cells(a1, a2, 1)
    H = np.zeros((cells.shape[0], norb, norb), dtype=np.complex128)
    h0 = _herm_random(rng, norb, 0.5)
    h0 = 0.5 * (h0 + h0.conj().T)
    # a gap: first atom's orbitals low, second atom's high
    diag = np.concatenate([rng.uniform(-4, -2, n0), rng.uniform(2, 4, n1)])
    np.fill_diagonal(h0, diag)
    H[0] = h0
    for p in range(npos):
        hr = _herm_random(rng, norb, 0.8)
        H[1 + p] = hr
        H[1 + npos + p] = hr.conj().T
    info = SystemInfo()
    info.ndim = 2
    info.filling = float(n0)
    info.bravaisLattice = np.array([a1, a2])
    info.motif = motif
    info.hamiltonian = H
    info.bravaisVectors = cells
    info.norbitals = np.array([n0, n1], dtype=np.int64)
    return SyntheticConfiguration(info, seed, f"random honeycomb {n0}+{n1} orbitals, seed={seed}")


def batch_workload(seed: int = 4242, count: int = 64):
    """The batched workload: ``count`` seeded random honeycomb models of 2-12 orbitals, k grids
    n x n with n drawn from {24, 36, 48, 60}, 1-3 valence and 1-3 conduction bands (as many as the
    model has on each side), r0 ~ U(5, 50) Angstrom, eps_s ~ U(1, 6), eps_m = 1, real-space Keldysh,
    direct term.  Returns a list of dicts (config, ncell, nv, nc, params)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        norb = int(rng.integers(2, 13))
        cfg = random_honeycomb(seed * 1000 + i, norb)
        n0 = int(cfg.systemInfo.filling)
        n1 = int(cfg.systemInfo.norbitals.sum()) - n0
        ncell = int(rng.choice([24, 36, 48, 60]))
        nv = int(rng.integers(1, min(3, n0) + 1))
        nc = int(rng.integers(1, min(3, n1) + 1))
        r0 = float(rng.uniform(5.0, 50.0))
        eps_s = float(rng.uniform(1.0, 6.0))
        out.append({"config": cfg, "ncell": ncell, "nv": nv, "nc": nc, "params": (1.0, eps_s, r0)})
    return out


def exciton_from_spec(spec, device: int = 0):
    """ExcitonTB of one batch_workload entry (mesh set, nothing on the device yet)."""
    from .exciton import ExcitonTB
    nv, nc = spec["nv"], spec["nc"]
    bands = list(range(-(nv - 1), 1)) + list(range(1, nc + 1))
    ex = ExcitonTB(spec["config"], spec["ncell"], 1, 0, spec["params"], bands=bands, device=device)
    ex.brillouinZoneMesh(spec["ncell"])
    return ex
