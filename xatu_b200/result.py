"""Results of the exciton solve: the reference's Result / ResultTB interface (Result.hpp, ResultTB.hpp).

Every quantity computed from the eigen-pairs -- kinetic energy, k-space weights, peak, spin, real-space
amplitudes, the envelope transform, oscillator strengths and the absorption spectrum -- is evaluated on the
device through the engine's C ABI (xatu_state_observables, xatu_realspace_amplitude, xatu_envelope_ft,
xatu_oscillator_strength, xatu_absorption).  This module keeps the reference's method names, arguments and
errors, and writes the reference's text formats (fprintf formats of Result.tpp / ResultTB.cpp, the columns of
skubo_w.f90) so existing plotting scripts read the files unchanged.

``textfile`` arguments take an open text file (anything with ``write``) or a path, which is then created.
"""
from __future__ import annotations

import contextlib
import ctypes
from typing import TYPE_CHECKING, Optional, Sequence, Union

import numpy as np

from . import _lib as L

if TYPE_CHECKING:  # pragma: no cover
    from .exciton import ExcitonTB

HARTREE = 27.211385

StateArg = Union[int, np.integer, np.ndarray, Sequence[complex]]


@contextlib.contextmanager
def _open(textfile):
    if hasattr(textfile, "write"):
        yield textfile
    else:
        with open(textfile, "w") as fh:
            yield fh


def generate_combinations(nvalues: int, ndim: int, centered: bool = False) -> np.ndarray:
    """Lattice::generateCombinations (Lattice.cpp:293-312): rows of ndim integers, dimension 0 fastest."""
    shift = nvalues // 2 if centered else 0
    vals = np.arange(nvalues, dtype=np.float64) - shift
    idx = np.arange(nvalues ** ndim)
    return np.stack([vals[(idx // nvalues ** d) % nvalues] for d in range(ndim)], axis=1)


def read_kubo_parameters(path: str = "kubo_w.in") -> dict:
    """get_kubo_parameters (skubo_w.f90:377-405): the seven values of kubo_w.in, each on the line after a
    comment line (Fortran list-directed reads: first token, 'd' exponents, optional quotes)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    if len(lines) < 13:
        raise ValueError(f"{path}: expected 13 lines (comment / value pairs and two file names)")

    def tok(i):
        t = lines[i].split()
        if not t:
            raise ValueError(f"{path}:{i + 1}: missing value")
        return t[0].strip("'\"")

    def num(i):
        return float(tok(i).replace("d", "e").replace("D", "e"))

    return {"w0": num(1), "wrange": num(3), "nw": int(num(5)), "eta": num(7), "broadening": tok(9),
            "file_sp": tok(11), "file_ex": tok(12)}


BROADENINGS = {"lorentzian": L.BROAD_LORENTZIAN, "gaussian": L.BROAD_GAUSSIAN, "exponential": L.BROAD_EXPONENTIAL}


class ResultTB:
    """Eigen-pairs of the BSE and their post-processing (Result.hpp, ResultTB.hpp).

    ``eigval``: exciton energies (eV); ``eigvec``: N x nstates coefficients (columns = states) in the
    e-h basis row k*nc*nv + c*nv + v of the exciton."""

    def __init__(self, exciton: "ExcitonTB", eigval: np.ndarray, eigvec: Optional[np.ndarray]):
        self.exciton = exciton
        self.system = exciton.system
        self.eigval = eigval
        self.eigvec = eigvec

    # ------------------------------------------------------------------ helpers
    def _columns(self, state: StateArg) -> np.ndarray:
        """N x ns Fortran-ordered coefficients: an index picks a column of eigvec, arrays are taken as given."""
        if isinstance(state, (int, np.integer)):
            if self.eigvec is None:
                raise ValueError("the result holds no eigenvectors")
            if not 0 <= int(state) < self.eigvec.shape[1]:
                raise IndexError(f"state {int(state)} out of range (0..{self.eigvec.shape[1] - 1})")
            X = self.eigvec[:, [int(state)]]
        else:
            X = np.asarray(state, dtype=np.complex128)
            if X.ndim == 1:
                X = X[:, None]
        if X.shape[0] != self.exciton.excitonbasisdim:
            raise ValueError(f"coefficient vectors must have length {self.exciton.excitonbasisdim}")
        return np.asfortranarray(X, dtype=np.complex128)

    def _all_states(self) -> np.ndarray:
        if self.eigvec is None:
            raise ValueError("the result holds no eigenvectors")
        return np.asfortranarray(self.eigvec, dtype=np.complex128)

    def observables(self, states: Optional[StateArg] = None, spin: bool = False) -> dict:
        """Device reductions of xatu_state_observables for the given states (default: every stored state):
        kinetic (ns), kweight (ns x nk, sum_cv |A|^2), peak (ns, k index), and spin (ns x 3 complex:
        total, hole, electron) when requested."""
        X = self._all_states() if states is None else self._columns(states)
        ns = X.shape[1]
        nk = self.system.nk
        kin = np.zeros(ns)
        kw = np.zeros((ns, nk))
        peak = np.zeros(ns, dtype=np.int64)
        sp = np.zeros((ns, 3), dtype=np.complex128) if spin else None
        self.exciton._call("xatu_state_observables", ns, L.ptr(X), L.ptr(kin), L.ptr(kw), L.ptr(peak), L.ptr(sp))
        out = {"kinetic": kin, "kweight": kw, "peak": peak}
        if spin:
            out["spin"] = sp
        return out

    def _dk(self) -> float:
        kp = self.system.kpoints
        if kp.shape[0] < 2:
            raise IndexError("the reciprocal amplitude is normalised by |k1 - k0|: the mesh needs two k points")
        return float(np.linalg.norm(kp[1] - kp[0]))

    # ------------------------------------------------------------------ observables (Result.tpp:16-160)
    def kineticEnergy(self, stateindex: int) -> float:
        """Result::kineticEnergy (Result.tpp:25-40)."""
        return float(self.observables(stateindex)["kinetic"][0])

    def potentialEnergy(self, stateindex: int) -> float:
        """Result::potentialEnergy (Result.tpp:50-53): E - K."""
        return float(self.eigval[stateindex] - self.kineticEnergy(stateindex))

    def bindingEnergy(self, stateindex: int, gap: float = -1) -> float:
        """Result::bindingEnergy (Result.tpp:64-76): E - gap, the gap from determineGap when gap == -1."""
        if gap == -1:
            gap = self.determineGap()
        elif gap < 0:
            print("Provided gap value must be positive")
        return float(self.eigval[stateindex] - gap)

    def determineGap(self) -> float:
        """Result::determineGap (Result.tpp:84-93): E_c - E_v of the band edges used, at the ground state's peak."""
        k = self.findExcitonPeak(0)
        ex = self.exciton
        band_list = list(ex.valenceBands) + list(ex.conductionBands)
        iv = band_list.index(int(np.max(ex.valenceBands)))
        ic = band_list.index(int(np.min(ex.conductionBands)))
        ev = np.zeros((self.system.nk, len(band_list)))
        ex._call("xatu_bands_download", L.ptr(ev), None, None, None)
        return float(ev[k, ic] - ev[k, iv])

    def findExcitonPeak(self, stateindex: int) -> int:
        """Result::findExcitonPeak (Result.tpp:478-484): k index of the largest |coefficient|."""
        return int(self.observables(stateindex)["peak"][0])

    def ftExcitonEnvelope(self, stateindex: int, electron_position, hole_position) -> float:
        """Result::ftExcitonEnvelope (Result.tpp:101-128): Re sum_k |A_k|^2 exp(-i k.(re - rh))."""
        d = np.asarray(electron_position, dtype=np.float64) - np.asarray(hole_position, dtype=np.float64)
        return float(self.ftExcitonEnvelopes(stateindex, d[None, :])[0, 0])

    def ftExcitonEnvelopes(self, states: StateArg, separations: np.ndarray) -> np.ndarray:
        """ftExcitonEnvelope for many states and separations r_e - r_h at once: (ns, npoints)."""
        X = self._columns(states)
        d = np.ascontiguousarray(np.asarray(separations, dtype=np.float64).reshape(-1, 3))
        out = np.zeros((X.shape[1], d.shape[0]))
        self.exciton._call("xatu_envelope_ft", X.shape[1], L.ptr(X), d.shape[0], L.ptr(d), L.ptr(out))
        return out

    def spinX(self, state: StateArg) -> np.ndarray:
        """ResultTB::spinX (ResultTB.cpp:21-98): [total, hole, electron] Sz of one state (index or coefficients)."""
        return self.observables(state, spin=True)["spin"][0]

    def excitonOscillatorStrength(self) -> np.ndarray:
        """ResultTB::excitonOscillatorStrength (ResultTB.cpp:242-298) for the stored states: 3 x nstates."""
        return self.exciton.excitonOscillatorStrength(self._all_states())

    def boundingBoxBZ(self) -> float:
        """Result::boundingBoxBZ (Result.tpp:492-498): the larger of max kx and max ky of the mesh."""
        kp = self.system.kpoints
        return float(max(np.max(kp[:, 0]), np.max(kp[:, 1])))

    # ------------------------------------------------------------------ real-space amplitude
    def realSpaceAmplitudes(self, states: StateArg, holeIndex: int, holeCell, cells: np.ndarray) -> np.ndarray:
        """realSpaceWavefunction for every state, cell and electron atom: (ns, ncells, natoms)."""
        X = self._columns(states)
        cells = np.ascontiguousarray(np.asarray(cells, dtype=np.float64).reshape(-1, 3))
        hc = np.ascontiguousarray(np.asarray(holeCell, dtype=np.float64).reshape(3))
        out = np.zeros((X.shape[1], cells.shape[0], self.system.natoms))
        self.exciton._call("xatu_realspace_amplitude", X.shape[1], L.ptr(X), int(holeIndex), L.ptr(hc),
                           cells.shape[0], L.ptr(cells), L.ptr(out))
        return out

    def realSpaceWavefunction(self, BSEcoefs, electronIndex: int, holeIndex: int, eCell, hCell) -> float:
        """ResultTB::realSpaceWavefunction (ResultTB.cpp:310-357)."""
        if not 0 <= int(electronIndex) < self.system.natoms:
            raise IndexError("electron atom index out of range")
        out = self.realSpaceAmplitudes(np.asarray(BSEcoefs), holeIndex, hCell, np.asarray(eCell)[None, :])
        return float(out[0, 0, int(electronIndex)])

    def writeRealspaceAmplitude(self, state: StateArg, holeIndex: int, holeCell, textfile, ncells: int = 3):
        """ResultTB::writeRealspaceAmplitude (ResultTB.cpp:370-408): hole position, then x, y and the
        probability of every atom of the cells within |a1| * ncells, then '#'."""
        s = self.system
        hole = s.motif[holeIndex, :3] + np.asarray(holeCell, dtype=np.float64)
        radius = float(np.linalg.norm(s.bravaisLattice[0])) * ncells
        cells = s.truncateSupercell(self.exciton.ncell, radius)
        amp = self.realSpaceAmplitudes(state, holeIndex, holeCell, cells)[0]
        with _open(textfile) as fh:
            fh.write("%11.8f\t%11.8f\t%14.11f\n" % (hole[0], hole[1], 0.0))
            lines = []
            for ci in range(cells.shape[0]):
                for atom in range(s.natoms):
                    pos = s.motif[atom, :3] + cells[ci]
                    lines.append("%11.8f\t%11.8f\t%14.11f\n" % (pos[0], pos[1], amp[ci, atom]))
            fh.write("".join(lines))
            fh.write("#\n")

    # ------------------------------------------------------------------ k-space writers
    def _kweights(self, state: StateArg) -> np.ndarray:
        return self.observables(state)["kweight"][0]

    def writeReciprocalAmplitude(self, state: StateArg, textfile):
        """Result::writeReciprocalAmplitude (Result.tpp:160-179)."""
        coef = self._kweights(state) / self._dk()
        kp = self.system.kpoints
        with _open(textfile) as fh:
            fh.write("kx\tky\tkz\tProb.\n")
            fh.write("".join("%11.8f\t%11.8f\t%11.8f\t%11.8f\n" % (k[0], k[1], k[2], c) for k, c in zip(kp, coef)))
            fh.write("#\n")

    def _replicas(self, rows: int) -> np.ndarray:
        """Reciprocal-lattice displacements of the extended writers (Result.tpp:211-216)."""
        s = self.system
        comb = generate_combinations(3, s.ndim, True)
        return comb[:, :rows] @ s.reciprocalLattice[:rows]

    def writeExtendedReciprocalAmplitude(self, state: StateArg, textfile):
        """Result::writeExtendedReciprocalAmplitude (Result.tpp:200-226): every k and its images by
        reciprocal vectors (-1..1 per dimension) inside the box |kx|, |ky| < boundingBoxBZ."""
        coef = self._kweights(state) / self._dk()
        box = self.boundingBoxBZ()
        shifts = self._replicas(self.system.ndim)
        out = []
        for k, c in zip(self.system.kpoints, coef):
            for g in shifts:
                d = k + g
                if abs(d[0]) < box and abs(d[1]) < box:
                    out.append("%11.8f\t%11.8f\t%11.8f\t%11.8f\n" % (d[0], d[1], d[2], c))
        with _open(textfile) as fh:
            fh.write("".join(out))
            fh.write("#\n")

    def _phase_coefs(self, state: StateArg) -> np.ndarray:
        if len(self.exciton.valenceBands) + len(self.exciton.conductionBands) != 2:
            raise ValueError("writePhase requires only one valence and conduction bands")
        return self._columns(state)[:, 0]

    def writePhase(self, state: StateArg, textfile):
        """Result::writePhase (Result.tpp:240-260): modulus and argument of the coefficient of every k."""
        x = self._phase_coefs(state)
        kp = self.system.kpoints
        with _open(textfile) as fh:
            fh.write("kx\tky\tkz\tMod.\tArg.\n")
            fh.write("".join("%11.8f\t%11.8f\t%11.8f\t%11.8f\t%11.8f\n" % (k[0], k[1], k[2], abs(c), np.angle(c))
                             for k, c in zip(kp, x)))
            fh.write("#\n")

    def writeExtendedPhase(self, state: StateArg, textfile):
        """Result::writeExtendedPhase (Result.tpp:283-313): modulus / |k1 - k0| and argument on the images of
        the mesh inside the bounding box (the reference combines b1 and b2, so ndim >= 2)."""
        x = self._phase_coefs(state)
        if self.system.ndim < 2:
            raise IndexError("writeExtendedPhase combines two reciprocal vectors (ndim >= 2)")
        dk = self._dk()
        box = self.boundingBoxBZ()
        shifts = self._replicas(2)
        out = []
        for k, c in zip(self.system.kpoints, x):
            mod = abs(c) / dk
            ph = np.angle(c)
            for g in shifts:
                d = k + g
                if abs(d[0]) < box and abs(d[1]) < box:
                    out.append("%11.8f\t%11.8f\t%11.8f\t%11.8f\t%11.8f\n" % (d[0], d[1], d[2], mod, ph))
        with _open(textfile) as fh:
            fh.write("kx\tky\tkz\tMod.\tArg.\n")
            fh.write("".join(out))
            fh.write("#\n")

    # ------------------------------------------------------------------ eigen-pair writers
    def _check_n(self, n: int):
        if n > self.exciton.excitonbasisdim or n < 0:
            raise ValueError("Optional argument n must be a positive integer equal or below basisdim")

    def writeEigenvalues(self, textfile, n: int = 0):
        """Result::writeEigenvalues (Result.tpp:404-418)."""
        self._check_n(n)
        N = self.exciton.excitonbasisdim
        m = N if n == 0 else n
        if m > len(self.eigval):
            raise IndexError(f"{m} eigenvalues requested, {len(self.eigval)} stored")
        with _open(textfile) as fh:
            fh.write("%d\t" % N)
            fh.write("".join("%11.7f\t" % e for e in self.eigval[:m]))
            fh.write("\n")

    def writeStates(self, textfile, n: int = 0):
        """Result::writeStates (Result.tpp:426-449): the basis (k, v, c) then the coefficients of n states."""
        self._check_n(n)
        ex = self.exciton
        N = ex.excitonbasisdim
        m = N if n == 0 else n
        X = self._all_states()
        if m > X.shape[1]:
            raise IndexError(f"{m} states requested, {X.shape[1]} stored")
        kp = self.system.kpoints
        nv, nc = len(ex.valenceBands), len(ex.conductionBands)
        with _open(textfile) as fh:
            fh.write("%d\n" % N)
            rows = []
            for ik in range(self.system.nk):
                for ic in range(nc):
                    for iv in range(nv):
                        k = kp[ik]
                        rows.append("%11.7f\t%11.7f\t%11.7f\t%d\t%d\n"
                                    % (k[0], k[1], k[2], int(ex.valenceBands[iv]), int(ex.conductionBands[ic])))
            fh.write("".join(rows))
            for i in range(m):
                col = X[:, i]
                fh.write("".join("%11.7f\t%11.7f\t" % (c.real, c.imag) for c in col))
                fh.write("\n")

    def writeSpin(self, n: int, textfile):
        """Result::writeSpin (Result.tpp:456-470): index, then the real parts of spinX's total, hole and
        electron values under the reference's header."""
        self._check_n(n)
        m = self.exciton.excitonbasisdim if n == 0 else n
        X = self._all_states()
        if m > X.shape[1]:
            raise IndexError(f"{m} states requested, {X.shape[1]} stored")
        spin = self.observables(X[:, :m], spin=True)["spin"]
        with _open(textfile) as fh:
            fh.write("n\tSt\tSe\tSh\n")
            fh.write("".join("%d\t%11.7f\t%11.7f\t%11.7f\n" % (i, s[0].real, s[1].real, s[2].real)
                             for i, s in enumerate(spin)))

    # ------------------------------------------------------------------ absorption (skubo_w.f90:2-173)
    def absorptionSpectrum(self, w0: float = 1.0, wrange: float = 6.0, nw: int = 400, eta: float = 0.08,
                           broadening: str = "lorentzian", states: Optional[Sequence[int]] = None) -> dict:
        """The conductivities skubo_w computes, on the device: w (eV, nw), sigma_sp (nw x 3 x 3 complex),
        sigma_ex (nw x 3 x 3 real), vme_ex (3 x ns) and the energies of the states used -- every stored
        state, or the given indices (the reference sums over all N states of a full diagonalisation)."""
        X = None
        E = None
        ns = 0
        if self.eigvec is not None:
            idx = np.arange(self.eigvec.shape[1]) if states is None else np.asarray(states, dtype=np.int64)
            X = np.asfortranarray(self.eigvec[:, idx], dtype=np.complex128)
            E = np.ascontiguousarray(np.asarray(self.eigval)[idx], dtype=np.float64)
            ns = X.shape[1]
        sp = np.zeros((nw, 3, 3), dtype=np.complex128)
        sx = np.zeros((nw, 3, 3))
        vx = np.zeros((3, max(ns, 1)), dtype=np.complex128, order="F")
        self.exciton._call("xatu_absorption", ns, L.ptr(E), L.ptr(X), float(w0), float(wrange), int(nw), float(eta),
                           BROADENINGS.get(broadening, L.BROAD_OTHER), L.ptr(sp), L.ptr(sx), L.ptr(vx))
        w = np.array([(w0 + wrange / nw * i) / HARTREE for i in range(nw)]) * HARTREE
        return {"w": w, "sigma_sp": sp, "sigma_ex": sx, "vme_ex": vx[:, :ns],
                "energies": np.zeros(0) if E is None else E}

    def writeAbsorptionSpectrum(self, parameters: str = "kubo_w.in"):
        """ResultTB::writeAbsorptionSpectrum (ResultTB.cpp:412-461 -> skubo_w.f90:2-173): reads kubo_w.in and
        writes the single-particle (-Re sigma) and exciton (Re sigma, a blank line, then the energy and
        velocity matrix elements of every state) files it names."""
        prm = read_kubo_parameters(parameters)
        r = self.absorptionSpectrum(prm["w0"], prm["wrange"], prm["nw"], prm["eta"], prm["broadening"])
        fmt = lambda vals: "".join(" %24.16E" % v for v in vals) + "\n"
        with open(prm["file_sp"], "w") as fh:
            for i in range(prm["nw"]):
                fh.write(fmt([r["w"][i]] + list(-r["sigma_sp"][i].reshape(9).real)))
        with open(prm["file_ex"], "w") as fh:
            for i in range(prm["nw"]):
                fh.write(fmt([r["w"][i]] + list(r["sigma_ex"][i].reshape(9))))
            fh.write(" \n")
            E = r["energies"]
            V = r["vme_ex"]
            for n in range(len(E)):
                # the reference's last column repeats Im of the y component (skubo_w.f90:164-166)
                fh.write(fmt([E[n] / HARTREE * HARTREE, V[0, n].real, V[0, n].imag, V[1, n].real, V[1, n].imag,
                              V[2, n].real, V[1, n].imag]))
        return r
