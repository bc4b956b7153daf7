"""Python host API mirroring Xatu's ExcitonTB for the BSE build+solve path.

The classes keep the reference's method names and argument meanings so a
script written against the reference's C++ API reads the same:

    config  = SystemConfiguration("hBN.model")
    exciton = ExcitonTB(config, ncell=20, nbands=1, nrmbands=0, parameters=[1, 1, 10])
    exciton.brillouinZoneMesh(20)
    exciton.initializeHamiltonian()
    exciton.BShamiltonian()
    results = exciton.diagonalize("diag", nstates=3)

Every computation runs on the GPU through the engine's C ABI
(include/xatu_bse.h); numpy is used only to hold host arrays.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from .config import ExcitonConfiguration, SystemConfiguration
from .result import ResultTB


class SystemTB:
    """Tight-binding system (System.hpp / SystemTB.hpp / Lattice.hpp data)."""

    def __init__(self, config: SystemConfiguration):
        info = config.systemInfo
        self.ndim = int(info.ndim)
        self.bravaisLattice = np.ascontiguousarray(info.bravaisLattice, dtype=np.float64)
        self.motif = np.ascontiguousarray(info.motif, dtype=np.float64)
        self.orbitals = np.asarray(info.norbitals, dtype=np.int32)
        self.unitCellList = np.ascontiguousarray(info.bravaisVectors, dtype=np.float64)
        self.hamiltonianMatrices = np.ascontiguousarray(info.hamiltonian, dtype=np.complex128)
        self.overlapMatrices = (np.ascontiguousarray(info.overlap, dtype=np.complex128)
                                if info.overlap.size else None)
        self.filling = int(info.filling)
        self.fermiLevel = self.filling - 1
        self.natoms = self.motif.shape[0]
        self.basisdim = int(sum(int(self.orbitals[int(s)]) for s in self.motif[:, 3]))
        self.reciprocalLattice = L.reciprocal_lattice(self.ndim, self.bravaisLattice)
        self.a = float(np.linalg.norm(self.bravaisLattice[0]))
        self.kpoints = np.zeros((0, 3))
        self.meshBZ = np.zeros((0, 3))
        self.nk = 0
        self.factor = 1

    # Lattice::brillouinZoneMesh (Lattice.cpp:140-162)
    def brillouinZoneMesh(self, n: int):
        self.kpoints = L.mesh_mp(self.ndim, self.reciprocalLattice, n)
        self.meshBZ = self.kpoints.copy()
        self.nk = self.kpoints.shape[0]
        self.factor = 1

    # Lattice::reducedBrillouinZoneMesh (Lattice.cpp:172-197)
    def reducedBrillouinZoneMesh(self, n: int, factor: int):
        self.meshBZ = L.mesh_mp(self.ndim, self.reciprocalLattice, n * factor)
        self.kpoints = L.mesh_reduced(self.ndim, self.reciprocalLattice, n, factor)
        self.nk = self.kpoints.shape[0]
        self.factor = factor

    # Lattice::shiftBZ (Lattice.cpp:203-220)
    def shiftBZ(self, shift: Sequence[float]):
        shift = np.asarray(shift, dtype=np.float64)
        if shift.size != 3:
            raise ValueError("shift vector must be 3d")
        if self.nk == 0:
            raise ValueError("To call this method kpoints must be initiallized first")
        self.kpoints = self.kpoints + shift[None, :]

    def findEquivalentPointBZ(self, kpoint, ncell: int) -> int:
        return int(L.equivalent_points(self.ndim, self.reciprocalLattice, ncell * self.factor,
                                       np.asarray(kpoint, dtype=np.float64))[0])

    def truncateSupercell(self, ncell: int, radius: float) -> np.ndarray:
        return L.truncate_supercell(self.ndim, self.bravaisLattice, ncell, radius)


class ExcitonTB:
    """B200 engine behind the reference's ExcitonTB interface (ExcitonTB.hpp:23-156)."""

    def __init__(self, system, ncell: int = 20, nbands: int = 1, nrmbands: int = 0,
                 parameters: Sequence[float] = (1, 5, 1), Q: Sequence[float] = (0., 0., 0.), *,
                 bands: Optional[Sequence[int]] = None, exciton_config: Optional[ExcitonConfiguration] = None,
                 device: int = 0):
        if hasattr(system, "systemInfo"):
            system = SystemTB(system)
        self.system: SystemTB = system
        self.device = device
        self._ctx = None
        self.gauge = "lattice"
        self.mode = "realspace"
        self.potential = "keldysh"
        self.exchangePotential = "keldysh"
        self.nReciprocalVectors = 1
        self.regularization = 0.0
        self.scissor = 0.0
        self.exchange = False
        if exciton_config is not None:
            self._init_from_config(exciton_config)
        else:
            self._init_attributes(ncell, parameters, Q)
            fl = self.system.fermiLevel
            if bands is not None:
                self._set_band_vector(np.asarray(bands, dtype=np.int64))
            else:
                if 2 * nbands > self.system.basisdim:
                    raise ValueError("Error: Number of bands cannot be higher than actual material bands")
                self.valenceBands = np.arange(fl - nbands - nrmbands + 1, fl - nrmbands + 1, dtype=np.int64)
                self.conductionBands = np.arange(fl + 1 + nrmbands, fl + nbands + nrmbands + 1, dtype=np.int64)
                self.bands = np.concatenate([self.valenceBands, self.conductionBands]) - fl
        self.HBS_built = None
        self._precision = None

    # ExcitonTB::initializeExcitonAttributes (ExcitonTB.cpp:20-34)
    def _init_attributes(self, ncell, parameters, Q):
        self.ncell = int(ncell)
        self.Q = np.asarray(Q, dtype=np.float64)
        self.eps_m, self.eps_s, self.r0 = (float(x) for x in parameters)
        self.cutoff = self.ncell / 2.5
        if self.r0 == 0:
            raise ValueError("Error: r0 must be non-zero")

    def _set_band_vector(self, bands: np.ndarray):
        fl = self.system.fermiLevel
        self.bands = bands
        self.valenceBands = bands[bands <= 0] + fl
        self.conductionBands = bands[bands > 0] + fl

    # ExcitonTB::initializeExcitonAttributes(cfg) (ExcitonTB.cpp:42-80)
    def _init_from_config(self, cfg: ExcitonConfiguration):
        info = cfg.excitonInfo
        bands = info.bands
        if bands.size == 0:
            bands = np.arange(-info.nbands + 1, info.nbands + 1, dtype=np.int64)
        self._init_attributes(info.ncell, [info.eps[0], info.eps[1], info.eps[2]], info.Q)
        self._set_band_vector(np.asarray(bands, dtype=np.int64))
        self.exchange = bool(info.exchange)
        self.scissor = float(info.scissor)
        self.mode = info.mode
        self.nReciprocalVectors = int(info.nReciprocalVectors)
        self.regularization = float(info.regularization) or self.system.a
        self.potential = info.potential
        self.exchangePotential = info.exchangePotential

    # ------------------------------------------------------------ setters (ExcitonTB.cpp:221-300, Exciton.tpp:16-117)
    def setParameters(self, *args):
        vals = args[0] if len(args) == 1 else args
        if len(vals) != 3:
            raise ValueError("parameters array must be 3d (eps_m, eps_s, r0)")
        self.eps_m, self.eps_s, self.r0 = (float(x) for x in vals)

    def setGauge(self, gauge: str):
        if gauge not in ("lattice", "atomic"):
            raise ValueError("setGauge(): gauge must be either lattice or atomic")
        self.gauge = gauge

    def setMode(self, mode: str):
        if mode not in ("realspace", "reciprocalspace"):
            raise ValueError("setMode(): mode must be either realspace or reciprocalspace")
        self.mode = mode

    def setReciprocalVectors(self, n: int):
        if n < 0:
            raise ValueError("setReciprocalVectors(): given number must be positive")
        self.nReciprocalVectors = int(n)

    def setRegularization(self, r: float):
        self.regularization = float(r)

    def setCutoff(self, cutoff: float):
        if cutoff > 0:
            self.cutoff = float(cutoff)

    def setScissor(self, shift: float):
        self.scissor = float(shift)

    def setExchange(self, exchange: bool):
        self.exchange = bool(exchange)

    def setQ(self, Q):
        Q = np.asarray(Q, dtype=np.float64)
        if Q.size == 3:
            self.Q = Q

    def setUnitCells(self, ncell: int):
        if ncell > 0:
            self.ncell = int(ncell)

    def brillouinZoneMesh(self, n: int):
        self.system.brillouinZoneMesh(n)

    # ------------------------------------------------------------ engine context
    @property
    def ctx(self):
        if self._ctx is None:
            c = ctypes.c_void_p()
            L.check(L.lib().xatu_ctx_create(ctypes.byref(c), self.device))
            self._ctx = c
        return self._ctx

    def close(self):
        if self._ctx is not None:
            L.lib().xatu_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name: str, *args):
        L.check(getattr(L.lib(), name)(self.ctx, *args), self.ctx)

    @property
    def excitonbasisdim(self) -> int:
        return self.system.nk * len(self.valenceBands) * len(self.conductionBands)

    # ------------------------------------------------------------ hot path
    def descriptors(self):
        """(system descriptor, exciton descriptor, kept arrays) of the ABI for this exciton: the
        checks and defaults of ExcitonTB::initializeHamiltonian (ExcitonTB.cpp:794-815)."""
        s = self.system
        if len(self.valenceBands) + len(self.conductionBands) == 0:
            raise ValueError("Error: Exciton object must have some bands")
        if s.nk == 0:
            raise ValueError("Error: BZ mesh must be initialized first")
        if self.regularization < 1e-10:
            self.regularization = s.a
        self.totalCells = (self.ncell * s.factor) ** s.ndim
        keep = {}
        keep["brav"] = np.ascontiguousarray(s.bravaisLattice)
        keep["motif"] = np.ascontiguousarray(s.motif)
        keep["orb"] = np.ascontiguousarray(s.orbitals, dtype=np.int32)
        keep["cells"] = np.ascontiguousarray(s.unitCellList)
        keep["ham"] = np.ascontiguousarray(s.hamiltonianMatrices)
        keep["ovl"] = None if s.overlapMatrices is None else np.ascontiguousarray(s.overlapMatrices)
        sd = L.SystemDesc(s.ndim, L.ptr(keep["brav"]), s.natoms, L.ptr(keep["motif"]), len(keep["orb"]),
                          L.ptr(keep["orb"]), keep["cells"].shape[0], L.ptr(keep["cells"]), L.ptr(keep["ham"]),
                          L.ptr(keep["ovl"]), s.filling, -1, 0)
        keep["kp"] = np.ascontiguousarray(s.kpoints, dtype=np.float64)
        keep["mesh"] = np.ascontiguousarray(s.meshBZ, dtype=np.float64)
        keep["vb"] = np.ascontiguousarray(self.valenceBands, dtype=np.int32)
        keep["cb"] = np.ascontiguousarray(self.conductionBands, dtype=np.int32)
        pot = {"keldysh": L.POT_KELDYSH, "coulomb": L.POT_COULOMB}
        ed = L.ExcitonDesc(self.ncell, s.factor, s.nk, L.ptr(keep["kp"]), keep["mesh"].shape[0],
                           L.ptr(keep["mesh"]), len(keep["vb"]), len(keep["cb"]), L.ptr(keep["vb"]),
                           L.ptr(keep["cb"]), self.eps_m, self.eps_s, self.r0, self.regularization, self.cutoff,
                           (ctypes.c_double * 3)(*self.Q), self.scissor, int(self.exchange),
                           L.MODE_REALSPACE if self.mode == "realspace" else L.MODE_RECIPROCAL,
                           self.nReciprocalVectors, pot[self.potential], pot[self.exchangePotential],
                           L.GAUGE_LATTICE if self.gauge == "lattice" else L.GAUGE_ATOMIC)
        return sd, ed, keep

    def initializeHamiltonian(self):
        """ExcitonTB::initializeHamiltonian (ExcitonTB.cpp:794-815): uploads the
        system and parameters, then runs the band solve and interaction tables on
        the device."""
        sd, ed, keep = self.descriptors()
        self._call("xatu_system_upload", ctypes.byref(sd))
        self._call("xatu_exciton_set", ctypes.byref(ed))
        self._call("xatu_bands_compute")
        self._call("xatu_interaction_build")
        self._precision = None

    def upload_bands(self, eigval, eigvec, eigvalQ=None, eigvecQ=None):
        """Replace the device band stacks with caller-supplied ones (gauge-controlled parity)."""
        ev = np.ascontiguousarray(eigval, dtype=np.float64)
        vv = np.ascontiguousarray(eigvec, dtype=np.complex128)
        evq = None if eigvalQ is None else np.ascontiguousarray(eigvalQ, dtype=np.float64)
        vvq = None if eigvecQ is None else np.ascontiguousarray(eigvecQ, dtype=np.complex128)
        self._call("xatu_bands_upload", L.ptr(ev), L.ptr(vv), L.ptr(evq), L.ptr(vvq))

    def bandStacks(self):
        nk, nb, norb = self.system.nk, len(self.valenceBands) + len(self.conductionBands), self.system.basisdim
        ev = np.zeros((nk, nb)); evq = np.zeros((nk, nb))
        vv = np.zeros((nk, nb, norb), dtype=np.complex128); vvq = np.zeros_like(vv)
        self._call("xatu_bands_download", L.ptr(ev), L.ptr(vv), L.ptr(evq), L.ptr(vvq))
        return ev, vv, evq, vvq

    def motifFT(self):
        na = self.system.natoms
        rows = self.system.meshBZ.shape[0]
        ft = np.zeros((rows, na, na), dtype=np.complex128)
        fq = np.zeros((na, na), dtype=np.complex128)
        if self.mode != "realspace":
            raise ValueError("motif FT table exists in real-space mode only")
        self._call("xatu_motif_ft_download", L.ptr(ft), L.ptr(fq))
        return ft, fq

    def BShamiltonian(self, precision: str = "fp64"):
        """ExcitonTB::BShamiltonian (ExcitonTB.cpp:822-921): assemble H on the device.

        precision "fp64": complex128 H (the reference's HBS_).  "mixed": FP64
        band-energy diagonal + split-BF16 interaction kernel for the tensor-core
        Davidson solver."""
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        self._call("xatu_bse_build", prec)
        self._precision = precision

    def BShamiltonianBasis(self, basis, precision: str = "fp64"):
        """ExcitonTB::BShamiltonian(const arma::imat& basis): H over the given e-h states,
        rows {valence band, conduction band, k index} (absolute band numbers)."""
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        b = np.ascontiguousarray(np.asarray(basis, dtype=np.int32).reshape(-1, 3))
        self._call("xatu_bse_build_basis", prec, b.shape[0], L.ptr(b))
        self._precision = precision

    @property
    def HBS(self) -> np.ndarray:
        """The assembled matrix copied to the host (row-major complex128)."""
        n = ctypes.c_int64()
        self._call("xatu_bse_dim", ctypes.byref(n))
        H = np.zeros((n.value, n.value), dtype=np.complex128)
        self._call("xatu_bse_copy_to_host", L.ptr(H))
        return H

    def diagonalize(self, method: str = "diag", nstates: int = 8, *, vectors: bool = True) -> ResultTB:
        """ExcitonTB::diagonalize (ExcitonTB.cpp:930-972).

        "diag": all eigenpairs, FP64 (needs the FP64 build); the result keeps
        the lowest ``nstates`` eigenvectors and all eigenvalues.  "davidson" /
        "sparse": lowest ``nstates`` by the device block Davidson."""
        n = ctypes.c_int64()
        self._call("xatu_bse_dim", ctypes.byref(n))
        N = n.value
        if method == "diag":
            ev = np.zeros(N)
            vec = np.zeros((nstates, N), dtype=np.complex128) if vectors else None
            self._call("xatu_bse_solve", L.SOLVER_DENSE_FP64, nstates, L.ptr(ev), L.ptr(vec))
            return ResultTB(self, ev, None if vec is None else vec.T.copy())
        if method in ("davidson", "sparse"):
            ev = np.zeros(nstates)
            vec = np.zeros((nstates, N), dtype=np.complex128) if vectors else None
            self._call("xatu_bse_solve", L.SOLVER_DAVIDSON, nstates, L.ptr(ev), L.ptr(vec))
            return ResultTB(self, ev, None if vec is None else vec.T.copy())
        raise ValueError(f"unknown method {method}")

    def excitonOscillatorStrength(self, eigvec: np.ndarray) -> np.ndarray:
        """ResultTB::excitonOscillatorStrength (ResultTB.cpp:242-298): 3 x nstates velocity
        matrix elements (atomic units) of the excitons in the columns of ``eigvec``."""
        X = np.asfortranarray(np.asarray(eigvec, dtype=np.complex128))
        if X.ndim == 1:
            X = X[:, None]
        out = np.zeros((3, X.shape[1]), dtype=np.complex128, order="F")
        self._call("xatu_oscillator_strength", X.shape[1], L.ptr(X), L.ptr(out))
        return out

    def adjointGradients(self, eigvec: np.ndarray, hamiltonian: bool = True, params: bool = True) -> dict:
        """Hellmann-Feynman gradients of the exciton energies of the normalised eigenvectors in the
        columns of ``eigvec`` (at most 8), through bands, interaction tables and assembly.

        Returns ``{"hamiltonian": G, "r0": ..., "eps_m": ..., "eps_s": ...}``: G has shape
        (nstates, nR, norb, norb) with G[n, R] = dE_n/dRe H(R) + i dE_n/dIm H(R) for perturbations that keep
        H(k) Hermitian (dE = Re sum conj(G) dH); the others have shape (nstates,)."""
        X = np.asfortranarray(np.asarray(eigvec, dtype=np.complex128))
        if X.ndim == 1:
            X = X[:, None]
        ns = X.shape[1]
        s = self.system
        G = np.zeros((ns, s.hamiltonianMatrices.shape[0], s.basisdim, s.basisdim), dtype=np.complex128) \
            if hamiltonian else None
        P = np.zeros((ns, 3)) if params else None
        self._call("xatu_adjoint", ns, L.ptr(X), L.ptr(G) if G is not None else None,
                   L.ptr(P) if P is not None else None)
        out = {}
        if G is not None:
            out["hamiltonian"] = G
        if P is not None:
            out["r0"], out["eps_m"], out["eps_s"] = P[:, 0].copy(), P[:, 1].copy(), P[:, 2].copy()
        return out

    def oscillatorWindowGradient(self, e_lo: float, e_hi: float, gradient: bool = True,
                                 hamiltonian: bool = False) -> dict:
        """Summed oscillator strength F of the excitons with e_lo <= E <= e_hi (FP64 build needed) and its
        gradients: {"F", "nwindow", "r0", "eps_m", "eps_s"} and, with hamiltonian=True, "hamiltonian"
        (nR x norb x norb, dF = Re sum conj(G) dH for Hermitian-consistent perturbations)."""
        nw = ctypes.c_int()
        F = ctypes.c_double()
        g = np.zeros(3)
        s = self.system
        G = np.zeros((s.hamiltonianMatrices.shape[0], s.basisdim, s.basisdim), dtype=np.complex128) \
            if hamiltonian else None
        self._call("xatu_oscillator_window_gradient", float(e_lo), float(e_hi), ctypes.byref(nw), ctypes.byref(F),
                   L.ptr(g) if gradient else None, L.ptr(G) if G is not None else None)
        out = {"F": F.value, "nwindow": nw.value}
        if gradient:
            out["r0"], out["eps_m"], out["eps_s"] = float(g[0]), float(g[1]), float(g[2])
        if G is not None:
            out["hamiltonian"] = G
        return out

    def davidsonConfig(self, tol: float = 0.0, max_iter: int = 0, block: int = 0):
        self._call("xatu_davidson_config", float(tol), int(max_iter), int(block))

    def setHxBackend(self, backend: str):
        """K.X kernel of the mixed build: "auto", "cuda" (CUDA cores) or "tc" (tcgen05 tensor cores)."""
        self._call("xatu_hx_backend", {"auto": 0, "cuda": 1, "tc": 2}[backend])

    def setBandsBackend(self, backend: str):
        """Band solve: "auto", "full" (every eigenpair of H(k), Jacobi) or "window" (the band list only)."""
        self._call("xatu_bands_backend", {"auto": 0, "full": 1, "window": 2}[backend])

    def matvec(self, X: np.ndarray) -> np.ndarray:
        """H X on the device with the current build (X: N x nvec complex)."""
        X = np.asarray(X, dtype=np.complex128)
        if X.ndim == 1:
            X = X[:, None]
        Xc = np.asfortranarray(X)
        Y = np.zeros_like(Xc, order="F")
        self._call("xatu_kernel_matvec", X.shape[1], L.ptr(Xc), L.ptr(Y))
        return Y

    def davidsonStats(self):
        it = ctypes.c_int()
        res = ctypes.c_double()
        self._call("xatu_davidson_stats", ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value

    def stageTimes(self):
        ms = (ctypes.c_float * 4)()
        self._call("xatu_stage_times", ms)
        return {"bands": ms[0], "tables": ms[1], "assembly": ms[2], "solve": ms[3]}

    def kernelStats(self, which: str):
        """(launches, total device ms, path) of "assembly", "hx" (path 1 CUDA cores, 2 tcgen05), "adjoint"
        (the last adjoint call) or "adjoint_pair" (its pair kernel)."""
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        path = ctypes.c_int()
        self._call("xatu_kernel_stats", {"assembly": 0, "hx": 1, "adjoint": 2, "adjoint_pair": 3}[which], ctypes.byref(n), ctypes.byref(ms),
                   ctypes.byref(path))
        return n.value, ms.value, path.value

    def kernelLaunches(self) -> int:
        n = ctypes.c_int64()
        self._call("xatu_kernel_launches", ctypes.byref(n))
        return n.value


def detectDegeneracies(eigval, n: int, precision: int):
    """detectDegeneracies (utils.cpp:121-154): [(energy, degeneracy), ...]."""
    if n < 0:
        raise ValueError("detectDegeneracies: n must be a positive integer")
    if n > len(eigval):
        raise ValueError("detectDegeneracies: n must be lower than total number of eigenstates")
    pairs = []
    prev = eigval[0]
    deg = 1
    thr = 10.0 ** (-precision)
    for i in range(1, n):
        e = eigval[i]
        if abs(e - prev) < thr:
            deg += 1
        else:
            pairs.append((float(prev), deg))
            deg = 1
        prev = e
    pairs.append((float(prev), deg))
    return pairs
