"""CPU oracle for the BSE build+solve path -- TEST INFRASTRUCTURE ONLY.

This module restates, on the CPU in FP64, the reference algorithm of Xatu
v1.3.1 for the exciton hot path:

    brillouinZoneMesh -> initializeHamiltonian -> BShamiltonian -> diagonalize

It is the checker for the CUDA engine.  Only ``tests/``, the smoke check in
``__graft_entry__`` and the CPU-baseline leg of ``bench.py`` import it; the
product package never does.

Split of the work:
  * geometry (Lattice.cpp), Bloch Hamiltonian and band solve (SystemTB.cpp),
    basis (Exciton.tpp) and the final eigensolve: numpy, below;
  * the potentials, motif lattice Fourier transform and the element-by-element
    BSE assembly (ExcitonTB.cpp:306-921): plain C with OpenMP in
    ``xatu_oracle.c`` (compiled by ``oracle/build.py`` into
    ``oracle/_build/liboracle.so``).

Third-party arithmetic: the reference calls LAPACK through Armadillo
(``eig_sym`` = zheevd, divide and conquer).  numpy.linalg.eigh is LAPACK
zheevd as well.  The eigen-solver versions of the reference are not pinned
(``README.md`` installs distribution packages); parity of the solve is pinned
through the golden exciton energies of the reference's ``test/tests.cpp``.

Pinned: ``tests/test_oracle_golden.py`` reproduces the reference's golden
energies (hBN realspace/reciprocal, spinful hBN, MoS2 energies, Q dispersion,
exchange and reduced-BZ cases) and its k-space wavefunction hash.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

PI = 3.141592653589793
_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def lib():
    """Load (building on first use if needed) the C part of the oracle."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from . import build as _b  # type: ignore
            _b.build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_stvh0.restype = ctypes.c_double
        L.orc_stvh0.argtypes = [ctypes.c_double]
        L.orc_keldysh.restype = ctypes.c_double
        L.orc_keldysh.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_coulomb.restype = ctypes.c_double
        L.orc_coulomb.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_keldysh_ft.restype = ctypes.c_double
        L.orc_keldysh_ft.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_motif_ft_stack.restype = None
        L.orc_motif_ft_stack.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_find_equivalent.restype = ctypes.c_int
        L.orc_find_equivalent.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p]
        L.orc_bse_build.restype = None
        L.orc_bse_build.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_bse_build_rows.restype = None
        L.orc_bse_build_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p]
        _lib = L
    return _lib


class _Params(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("natoms", ctypes.c_int), ("norb", ctypes.c_int),
                ("motif", ctypes.c_void_p), ("orb_offset", ctypes.c_void_p),
                ("a1norm", ctypes.c_double), ("b1norm", ctypes.c_double),
                ("unit_cell_area", ctypes.c_double), ("eps_m", ctypes.c_double),
                ("eps_s", ctypes.c_double), ("r0", ctypes.c_double),
                ("regularization", ctypes.c_double), ("cutoff", ctypes.c_double),
                ("total_cells", ctypes.c_double)]


class _BseInput(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("basis_v", ctypes.c_void_p), ("basis_c", ctypes.c_void_p),
                ("basis_k", ctypes.c_void_p), ("nk", ctypes.c_int), ("nb", ctypes.c_int),
                ("kpoints", ctypes.c_void_p), ("eigvec", ctypes.c_void_p), ("eigvecQ", ctypes.c_void_p),
                ("eigval", ctypes.c_void_p), ("eigvalQ", ctypes.c_void_p), ("scissor", ctypes.c_double),
                ("exchange", ctypes.c_int), ("mode", ctypes.c_int), ("ft_stack", ctypes.c_void_p),
                ("ft_Q", ctypes.c_void_p), ("recip", ctypes.c_void_p), ("inv_recip", ctypes.c_void_p),
                ("n_eff", ctypes.c_int), ("nG", ctypes.c_int), ("G", ctypes.c_void_p),
                ("Q", ctypes.c_double * 3)]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ----------------------------------------------------------------------------- geometry


def reciprocal_lattice(bravais: np.ndarray, ndim: int) -> np.ndarray:
    """Lattice::calculateReciprocalLattice (Lattice.cpp:56-80)."""
    bravais = np.asarray(bravais, dtype=np.float64)
    if ndim == 1:
        return 2.0 * PI * bravais / np.linalg.norm(bravais) ** 2
    coef = bravais[:, :ndim]
    out = np.zeros((ndim, 3))
    for i in range(ndim):
        rhs = np.zeros(ndim)
        rhs[i] = 2 * PI
        out[i, :ndim] = np.linalg.solve(coef, rhs)
    return out


def unit_cell_area(bravais: np.ndarray, ndim: int) -> float:
    """Lattice::computeUnitCellArea (Lattice.cpp:119-131)."""
    if ndim == 1:
        return float(np.linalg.norm(bravais[0]))
    cross = np.cross(bravais[0], bravais[1])
    if ndim == 2:
        return float(np.linalg.norm(cross))
    return float(np.dot(cross, bravais[2]))


def generate_combinations(nvalues: int, ndim: int, centered: bool = False) -> np.ndarray:
    """Lattice::generateCombinations (Lattice.cpp:293-312): dimension 0 varies fastest."""
    shift = nvalues // 2 if centered else 0
    return _combinations(np.arange(nvalues, dtype=np.float64) - shift, ndim)


def _combinations(vals: np.ndarray, ndim: int) -> np.ndarray:
    n = len(vals)
    total = n ** ndim
    out = np.zeros((total, ndim))
    idx = np.arange(total)
    for d in range(ndim):
        out[:, d] = vals[(idx // n ** d) % n]
    return out


def brillouin_zone_mesh(recip: np.ndarray, ndim: int, n: int) -> np.ndarray:
    """Lattice::brillouinZoneMesh (Lattice.cpp:140-162)."""
    comb = _combinations(np.arange(n, dtype=np.float64), ndim)
    if n % 2 == 1:
        comb = comb + 0.5
    k = np.zeros((n ** ndim, 3))
    for i in range(n ** ndim):
        kp = np.zeros(3)
        for j in range(ndim):
            kp = kp + (2 * comb[i, j] - n) / (2 * n) * recip[j]
        k[i] = kp
    return k


def reduced_brillouin_zone_mesh(recip: np.ndarray, ndim: int, n: int, factor: int):
    """Lattice::reducedBrillouinZoneMesh (Lattice.cpp:172-197) -> (kpoints, meshBZ)."""
    mesh = brillouin_zone_mesh(recip, ndim, n * factor)
    comb = _combinations(np.arange(n, dtype=np.float64), ndim)
    if n % 2 == 1:
        comb = comb + 0.5
    k = np.zeros((n ** ndim, 3))
    for i in range(n ** ndim):
        kp = np.zeros(3)
        for j in range(ndim):
            kp = kp + (2 * comb[i, j] - n) / (2 * n * factor) * recip[j]
        k[i] = kp
    return k, mesh


def truncate_supercell(bravais: np.ndarray, ndim: int, ncell: int, radius: float) -> np.ndarray:
    """Lattice::truncateSupercell (Lattice.cpp:320-341)."""
    comb = _combinations(np.arange(ncell, dtype=np.float64) - ncell // 2, ndim)
    cells = []
    for i in range(comb.shape[0]):
        v = np.zeros(3)
        for j in range(ndim):
            v = v + comb[i, j] * bravais[j]
        if np.linalg.norm(v) < radius + 1e-5:
            cells.append(v)
    return np.array(cells).reshape(-1, 3)


def truncate_reciprocal_supercell(recip: np.ndarray, ndim: int, ncell: int, radius: float) -> np.ndarray:
    """Lattice::truncateReciprocalSupercell (Lattice.cpp:349-370)."""
    return truncate_supercell(recip, ndim, ncell, radius)


def inverse_reciprocal_matrix(recip: np.ndarray) -> np.ndarray:
    """Lattice::calculateInverseReciprocalMatrix (Lattice.cpp:228-240)."""
    return np.linalg.inv(recip @ recip.T)


def find_equivalent_point(recip, inv, n_eff, kpoint) -> int:
    """Lattice::findEquivalentPointBZ (Lattice.cpp:251-279), C restatement."""
    ndim = recip.shape[0]
    r = np.ascontiguousarray(recip, dtype=np.float64)
    iv = np.ascontiguousarray(inv, dtype=np.float64)
    k = np.ascontiguousarray(kpoint, dtype=np.float64)
    return lib().orc_find_equivalent(ndim, _ptr(r), _ptr(iv), int(n_eff), _ptr(k))


# ----------------------------------------------------------------------------- system


@dataclass
class OracleSystem:
    """Arrays of a SystemTB (System.cpp:46-60, SystemTB.cpp:29-31)."""
    ndim: int
    bravais: np.ndarray          # ndim x 3
    motif: np.ndarray            # natoms x 4
    norbitals: np.ndarray        # per species
    cells_h: np.ndarray          # nR x 3
    hamiltonian: np.ndarray      # nR x norb x norb complex, [R][row][col]
    filling: int
    overlap: np.ndarray | None = None
    is_au: bool = False
    is_triangular: bool = field(init=False)

    def __post_init__(self):
        self.bravais = np.asarray(self.bravais, dtype=np.float64).reshape(-1, 3)
        self.motif = np.asarray(self.motif, dtype=np.float64).reshape(-1, 4)
        self.hamiltonian = np.asarray(self.hamiltonian, dtype=np.complex128)
        self.cells_h = np.asarray(self.cells_h, dtype=np.float64).reshape(-1, 3)
        self.recip = reciprocal_lattice(self.bravais, self.ndim)
        self.a = float(np.linalg.norm(self.bravais[0]))
        self.area = unit_cell_area(self.bravais, self.ndim)
        self.natoms = self.motif.shape[0]
        self.orb_per_atom = np.array([int(self.norbitals[int(s)]) for s in self.motif[:, 3]], dtype=np.int32)
        self.orb_offset = np.concatenate([[0], np.cumsum(self.orb_per_atom)]).astype(np.int32)
        self.basisdim = int(self.orb_offset[-1])
        self.fermi_level = int(self.filling) - 1
        h0 = self.hamiltonian[0]
        upper = np.allclose(np.tril(h0, -1), 0, atol=0, rtol=0)
        lower = np.allclose(np.triu(h0, 1), 0, atol=0, rtol=0)
        self.is_triangular = bool(upper != lower)  # utils.cpp:176-178

    def hamiltonian_k(self, k: np.ndarray) -> np.ndarray:
        """SystemTB::hamiltonian (SystemTB.cpp:60-75)."""
        ph = np.exp(1j * (self.cells_h @ k))
        h = np.tensordot(ph, self.hamiltonian, axes=(0, 0))
        if self.is_triangular:
            h = h - np.diag(np.diag(h) / 2)
            h = h + h.conj().T
        return h

    def overlap_k(self, k: np.ndarray) -> np.ndarray:
        """SystemTB::overlap (SystemTB.cpp:86-101)."""
        ph = np.exp(1j * (self.cells_h @ k))
        s = np.tensordot(ph, self.overlap, axes=(0, 0))
        if self.is_triangular:
            s = s - np.diag(np.diag(s) / 2)
            s = s + s.conj().T
        return s

    def solve_bands(self, k: np.ndarray):
        """SystemTB::solveBands (SystemTB.cpp:113-125) + Loewdin (:136-156)."""
        h = self.hamiltonian_k(k)
        if self.overlap is not None and len(self.overlap):
            if self.is_au:
                h = h * 27.2
            s = self.overlap_k(k)
            w, u = np.linalg.eigh(s)
            if np.any(w <= 0):
                raise ValueError("Zero or negative overlap eigenvalues found")
            x = (u * (1.0 / np.sqrt(w))) @ u.conj().T
            h = x @ h @ x
        return np.linalg.eigh(h)


def fix_global_phase(coefs: np.ndarray) -> np.ndarray:
    """ExcitonTB::fixGlobalPhase (ExcitonTB.cpp:673-683): column sum made real and positive."""
    sums = coefs.sum(axis=0)
    return coefs * np.exp(-1j * np.angle(sums))[None, :]


# ----------------------------------------------------------------------------- exciton


class OracleExciton:
    """ExcitonTB (ExcitonTB.cpp:20-34, :128-144) restated for the build+solve path."""

    def __init__(self, system: OracleSystem, ncell: int, nbands: int = 1, nrmbands: int = 0,
                 parameters=(1.0, 5.0, 1.0), Q=(0.0, 0.0, 0.0), bands=None):
        self.system = system
        self.ncell = ncell
        self.eps_m, self.eps_s, self.r0 = (float(x) for x in parameters)
        if self.r0 == 0:
            raise ValueError("r0 must be non-zero")
        self.Q = np.asarray(Q, dtype=np.float64)
        self.cutoff = ncell / 2.5
        self.scissor = 0.0
        self.exchange = False
        self.mode = "realspace"
        self.n_reciprocal = 1
        self.potential = "keldysh"
        self.exchange_potential = "keldysh"
        self.regularization = 0.0  # parametric constructors leave it unset (ExcitonTB.hpp:32)
        self.factor = 1
        fl = system.fermi_level
        if bands is None:
            self.valence = np.arange(fl - nbands - nrmbands + 1, fl - nrmbands + 1)
            self.conduction = np.arange(fl + 1 + nrmbands, fl + nbands + nrmbands + 1)
        else:
            bands = np.asarray(bands)
            self.valence = bands[bands <= 0] + fl
            self.conduction = bands[bands > 0] + fl
        self.band_list = np.concatenate([self.valence, self.conduction]).astype(np.int64)
        self.kpoints = None
        self.mesh = None

    # Exciton::brillouinZoneMesh -> Lattice::brillouinZoneMesh
    def brillouin_zone_mesh(self, n: int):
        self.kpoints = brillouin_zone_mesh(self.system.recip, self.system.ndim, n)
        self.mesh = self.kpoints
        self.factor = 1

    def reduced_brillouin_zone_mesh(self, n: int, factor: int):
        self.kpoints, self.mesh = reduced_brillouin_zone_mesh(self.system.recip, self.system.ndim, n, factor)
        self.factor = factor

    def shift_bz(self, shift):
        self.kpoints = self.kpoints + np.asarray(shift, dtype=np.float64)[None, :]

    def params(self) -> _Params:
        s = self.system
        self._keep = [np.ascontiguousarray(s.motif), np.ascontiguousarray(s.orb_offset)]
        return _Params(s.ndim, s.natoms, s.basisdim, _ptr(self._keep[0]), _ptr(self._keep[1]),
                       s.a, float(np.linalg.norm(s.recip[0])), s.area, self.eps_m, self.eps_s, self.r0,
                       self.regularization, self.cutoff, float(self.total_cells))

    def initialize_hamiltonian(self):
        """ExcitonTB::initializeHamiltonian (ExcitonTB.cpp:794-815) + initializeResultsH0 (:707-787)."""
        s = self.system
        if self.kpoints is None:
            raise ValueError("BZ mesh must be initialized first")
        if self.regularization < 1e-10:
            self.regularization = s.a
        nk = self.kpoints.shape[0]
        self.total_cells = (self.ncell * self.factor) ** s.ndim
        nv, nc = len(self.valence), len(self.conduction)
        # Exciton::createBasis (Exciton.tpp:128-147): row = ik*(nc*nv) + ic*nv + iv
        N = nk * nc * nv
        ik, ic, iv = np.meshgrid(np.arange(nk), np.arange(nc), np.arange(nv), indexing="ij")
        self.basis_k = ik.reshape(-1).astype(np.int32)
        self.basis_c = (nv + ic.reshape(-1)).astype(np.int32)   # stack column (bandToIndex)
        self.basis_v = iv.reshape(-1).astype(np.int32)
        self.N = N
        nb = len(self.band_list)
        self.eigval = np.zeros((nk, nb))
        self.eigvec = np.zeros((nk, nb, s.basisdim), dtype=np.complex128)
        self.eigvalQ = np.zeros((nk, nb))
        self.eigvecQ = np.zeros((nk, nb, s.basisdim), dtype=np.complex128)
        qnz = np.linalg.norm(self.Q) != 0
        for i in range(nk):
            w, u = s.solve_bands(self.kpoints[i])
            u = fix_global_phase(u)
            self.eigval[i] = w[self.band_list]
            self.eigvec[i] = u[:, self.band_list].T
            if qnz:
                w, u = s.solve_bands(self.kpoints[i] + self.Q)
                u = fix_global_phase(u)
                self.eigvalQ[i] = w[self.band_list]
                self.eigvecQ[i] = u[:, self.band_list].T
            else:
                self.eigvalQ[i] = self.eigval[i]
                self.eigvecQ[i] = self.eigvec[i]
        radius = s.a * self.cutoff
        self.cells = truncate_supercell(s.bravais, s.ndim, self.ncell, radius)
        self.inv_recip = inverse_reciprocal_matrix(s.recip)
        na = s.natoms
        self.ft_stack = np.zeros((self.mesh.shape[0], na, na), dtype=np.complex128)
        self.ft_Q = np.zeros((na, na), dtype=np.complex128)
        if self.mode == "realspace":
            self.ft_stack = self.motif_ft(self.potential, self.mesh)
        if self.exchange:
            self.ft_Q = self.motif_ft(self.exchange_potential, self.Q[None, :])[0]
        if self.mode == "reciprocalspace":
            rad = self.cutoff * float(np.linalg.norm(s.recip[0]))
            self.G = truncate_reciprocal_supercell(s.recip, s.ndim, self.n_reciprocal, rad)
        else:
            self.G = np.zeros((1, 3))

    def motif_ft(self, potential: str, q: np.ndarray) -> np.ndarray:
        kind = 1 if potential == "coulomb" else 0
        p = self.params()
        q = np.ascontiguousarray(q, dtype=np.float64)
        cells = np.ascontiguousarray(self.cells)
        out = np.zeros((q.shape[0], self.system.natoms, self.system.natoms), dtype=np.complex128)
        lib().orc_motif_ft_stack(ctypes.byref(p), kind, q.shape[0], _ptr(q), cells.shape[0], _ptr(cells),
                                 _ptr(out))
        return out

    def _bse_input(self):
        keep = dict(bv=np.ascontiguousarray(self.basis_v), bc=np.ascontiguousarray(self.basis_c),
                    bk=np.ascontiguousarray(self.basis_k), kp=np.ascontiguousarray(self.kpoints),
                    ev=np.ascontiguousarray(self.eigvec), evq=np.ascontiguousarray(self.eigvecQ),
                    el=np.ascontiguousarray(self.eigval), elq=np.ascontiguousarray(self.eigvalQ),
                    ft=np.ascontiguousarray(self.ft_stack), ftq=np.ascontiguousarray(self.ft_Q),
                    rec=np.ascontiguousarray(self.system.recip), inv=np.ascontiguousarray(self.inv_recip),
                    G=np.ascontiguousarray(self.G))
        inp = _BseInput(self.N, _ptr(keep["bv"]), _ptr(keep["bc"]), _ptr(keep["bk"]), self.kpoints.shape[0],
                        len(self.band_list), _ptr(keep["kp"]), _ptr(keep["ev"]), _ptr(keep["evq"]),
                        _ptr(keep["el"]), _ptr(keep["elq"]), self.scissor, int(self.exchange),
                        0 if self.mode == "realspace" else 1, _ptr(keep["ft"]), _ptr(keep["ftq"]),
                        _ptr(keep["rec"]), _ptr(keep["inv"]), self.ncell * self.factor, keep["G"].shape[0],
                        _ptr(keep["G"]), (ctypes.c_double * 3)(*self.Q))
        return inp, keep

    def bs_hamiltonian(self) -> np.ndarray:
        """ExcitonTB::BShamiltonian (ExcitonTB.cpp:840-921) -> full Hermitian H (row-major)."""
        p = self.params()
        inp, keep = self._bse_input()
        H = np.zeros((self.N, self.N), dtype=np.complex128)
        lib().orc_bse_build(ctypes.byref(p), ctypes.byref(inp), _ptr(H))
        self.H = H
        return H

    def bs_rows(self, row0: int, row1: int) -> np.ndarray:
        """Upper-triangle rows [row0, row1) of -(D - X) (bounded CPU-baseline sample)."""
        p = self.params()
        inp, keep = self._bse_input()
        out = np.zeros((row1 - row0, self.N), dtype=np.complex128)
        lib().orc_bse_build_rows(ctypes.byref(p), ctypes.byref(inp), row0, row1, _ptr(out))
        return out

    def diagonalize(self, method: str = "diag", nstates: int = 8):
        """ExcitonTB::diagonalizeRaw (ExcitonTB.cpp:930-959); 'diag' = LAPACK zheevd."""
        if method == "diag":
            return np.linalg.eigh(self.H)
        if method == "davidson":
            return davidson_method(self.H, nstates)
        raise ValueError(f"unsupported method {method}")


def davidson_method(mat: np.ndarray, neigval: int, tol: float = 1e-8, max_seconds: float = None,
                    stats: dict = None, check_hermitian: bool = True):
    """davidson_method (davidson.cpp:5-60), restated in numpy (QR by LAPACK geqrf).

    max_seconds (not in the reference): stop after the iteration that crosses this wall time, for bounded CPU
    timings; ``stats`` (a dict) then receives the iteration count and whether the eigenvalues converged.
    check_hermitian=False skips the reference's O(N^2) Hermiticity check for matrices built Hermitian."""
    import time as _time
    t_start = _time.perf_counter()
    n = mat.shape[0]
    max_it = n // 2
    k = neigval * 2
    if check_hermitian and not np.allclose(mat, mat.conj().T):
        raise ValueError("davidson_method: provided matrix must be hermitian")
    guess = np.eye(n, k, dtype=np.complex128)
    aux = np.ones(neigval)
    eigval = eigvec = None
    if stats is not None:
        stats.update(iterations=0, converged=False)
    for i in range(max_it):
        if stats is not None:
            stats["iterations"] = i + 1
        Qm, _ = np.linalg.qr(guess)
        proj = Qm.conj().T @ mat @ Qm
        eigval, eigvec = np.linalg.eigh(proj)
        eigvec = Qm[:, : (i + 1) * k] @ eigvec[:, :k]
        cols = [Qm]
        for j in range(k):
            w = mat @ eigvec[:, j] - eigval[j] * eigvec[:, j]
            cols.append((w / (eigval[j] - mat[j, j]))[:, None])
        Qm = np.concatenate(cols, axis=1)
        if np.linalg.norm(eigval[:neigval] - aux) < tol:
            if stats is not None:
                stats["converged"] = True
            break
        aux = eigval[:neigval].copy()
        guess = Qm
        if max_seconds is not None and _time.perf_counter() - t_start > max_seconds:
            break
    return eigval[:neigval], eigvec


# ----------------------------------------------------------------------------- utils


def detect_degeneracies(eigval, n: int, precision: int):
    """detectDegeneracies (utils.cpp:121-154)."""
    if n < 0 or n > len(eigval):
        raise ValueError("detectDegeneracies: bad n")
    pairs = []
    prev = eigval[0]
    deg = 1
    thr = 10.0 ** (-precision)
    for i in range(1, n):
        e = eigval[i]
        if abs(e - prev) < thr:
            deg += 1
        else:
            pairs.append((prev, deg))
            deg = 1
        prev = e
    pairs.append((prev, deg))
    return pairs


def array2hash(array, subview: bool = False) -> float:
    """array2hash (utils.hpp:62-78).  ``array`` keeps Armadillo's shape: a row
    vector is 1 x n, a column vector n x 1 (1-D input is taken as a column).

    With ``subview=True`` the weighted copy aliases the input, as it does in
    the reference when the argument is an Armadillo ``subview_row`` (e.g.
    ``bravaisLattice.row(i)`` in tests.cpp:40-51): ``T copyArray(array)`` is
    then a view of the same memory, so the |a| and nonzero terms see the
    weighted values."""
    a = np.asarray(array)
    if a.ndim == 1:
        a = a[:, None]
    i = np.arange(a.shape[0])[:, None]
    j = np.arange(a.shape[1])[None, :]
    cp = a * (i * j + j + 1)
    base = cp if subview else a
    h = (np.abs(base).sum() + (base != 0).sum() + (np.real(cp) * 1.5).sum() + (np.imag(cp) * 1.5).sum()
         + (np.imag(cp) * np.real(cp)).sum()) / a.size
    return float(h)


# ----------------------------------------------------------------------------- oscillator strengths

BOHR = 0.52917721067121
HARTREE = 27.211385


def vme_single_particle(system: OracleSystem, k_au: np.ndarray, C: np.ndarray, e_au: np.ndarray) -> np.ndarray:
    """Velocity matrix elements between the stored bands at one k (atomic units).

    Restates get_vme_kernels + get_eigen_vme (skubo_w.f90:445-628) with the
    hopping derivatives of hoppings_observables_TB (skubo_w.f90:407-443):
    only the lower triangle (a' <= a) of every kernel is summed over R (with
    R_z = 0), the upper triangle is filled by conjugation -- for the A kernel
    as conj(A_aa') + i conj(S'_aa'), which also overwrites its diagonal -- and
    the orbital positions enter through R index 0 only.  C: norb x nb band
    coefficients, e_au: nb band energies (Hartree).  Returns vme[3][nb][nb]."""
    norb = system.basisdim
    R = system.cells_h / BOHR
    H = system.hamiltonian / HARTREE                       # [R][a][a']
    S = np.zeros_like(H)
    if system.overlap is not None and len(system.overlap):
        S = np.real(system.overlap).astype(np.complex128)
    else:
        S[:] = np.eye(norb)[None, :, :]
    pos = np.zeros((norb, 3))
    for a in range(system.natoms):
        pos[system.orb_offset[a]:system.orb_offset[a + 1]] = system.motif[a, :3] / BOHR
    nR = R.shape[0]
    lower = np.tril(np.ones((norb, norb), dtype=bool))
    phase = np.exp(1j * (k_au[0] * R[:, 0] + k_au[1] * R[:, 1] + k_au[2] * 0.0))   # R_z = 0
    hk = np.einsum("r,rab->ab", phase, H)
    sk = np.einsum("r,rab->ab", phase, S)
    hder = np.zeros((3, norb, norb), dtype=np.complex128)
    sder = np.zeros((3, norb, norb), dtype=np.complex128)
    for nj, comp in ((0, R[:, 0]), (1, R[:, 1])):
        hder[nj] = np.einsum("r,rab->ab", phase * 1j * comp, H)
        sder[nj] = np.einsum("r,rab->ab", phase * 1j * comp, S)
    akern = np.zeros((3, norb, norb), dtype=np.complex128)
    for nj in range(3):
        # rhop(nj, R index 0, a, a) = position of orbital a
        akern[nj] = 1j * sder[nj] + np.diag(pos[:, nj]) * phase[0]
    # lower triangle kept, upper from conjugation
    hk_f = np.where(lower, hk, hk.T.conj())
    hder_f = np.where(lower[None], hder, np.transpose(hder, (0, 2, 1)).conj())
    for nj in range(3):
        np.fill_diagonal(hder_f[nj], np.diag(hder[nj]).conj())   # the mirror loop also conjugates the diagonal
    sder_l = np.where(lower[None], sder, 0)
    ak_f = np.where(lower[None], akern, np.transpose(akern, (0, 2, 1)).conj()
                    + 1j * np.transpose(sder_l, (0, 2, 1)).conj())
    # diagonal: overwritten by conj(A_aa) + i conj(S'_aa)
    for nj in range(3):
        d = np.diag(akern[nj]).conj() + 1j * np.diag(sder[nj]).conj()
        np.fill_diagonal(ak_f[nj], d)
    nb = C.shape[1]
    vme = np.zeros((3, nb, nb), dtype=np.complex128)
    for nn in range(nb):
        for nnp in range(nn + 1):
            cc = np.outer(C[:, nn].conj(), C[:, nnp])               # conj(amu) * amup  [a][a']
            for nj in range(3):
                va = np.sum(cc * hder_f[nj])
                vb = np.sum(cc * (e_au[nn] * ak_f[nj] - e_au[nnp] * ak_f[nj].T.conj())) * 1j
                vme[nj, nn, nnp] = va + vb
                vme[nj, nnp, nn] = np.conj(va + vb)
    return vme


def exciton_oscillator_strength(ex: "OracleExciton", eigvec: np.ndarray) -> np.ndarray:
    """ResultTB::excitonOscillatorStrength (ResultTB.cpp:242-298) with
    exciton_oscillator_strength (skubo_w.f90:175-330): returns vme_ex[3][nstates],
    vme_ex(nj, s) = sum_j X(j, s) vme(k_j, nj, v_j, c_j) (no conjugation of X).
    Unlike the reference, the exciton energies are not converted in place."""
    s = ex.system
    nv, nc = len(ex.valence), len(ex.conduction)
    nk = ex.kpoints.shape[0]
    v = np.zeros((3, ex.N), dtype=np.complex128)
    for ik in range(nk):
        C = ex.eigvec[ik].T                                         # norb x nb
        vme = vme_single_particle(s, ex.kpoints[ik] * BOHR, C, ex.eigval[ik] / HARTREE)
        for ic in range(nc):
            for iv in range(nv):
                j = ik * nc * nv + ic * nv + iv
                v[:, j] = vme[:, iv, nv + ic]
    return v @ eigvec
