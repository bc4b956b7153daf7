"""Readers for Xatu's plain-text input files.

``SystemConfiguration`` reads a ``.model`` tight-binding file and
``ExcitonConfiguration`` an exciton run file.  Both follow the reference's
block format (ConfigurationBase.cpp:43-150): a line containing ``#`` opens a
block whose key is the rest of the line, lower-cased with whitespace removed;
empty lines and lines containing ``!`` are skipped; ``,`` and ``;`` separate
values like blanks.  Matrices in a block are separated by ``&`` lines, complex
entries are written ``re +imj`` (SystemConfiguration.cpp:159-228).

The parsed fields keep the reference's names (``systemInfo`` /
``excitonInfo``) so code written against the reference reads the same.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np


def _parse_argument(line: str) -> str:
    """ConfigurationBase::parseArgument (ConfigurationBase.cpp:43-50)."""
    s = line[line.find("#") + 1:]
    return "".join(s.split()).lower()


def _standarize(line: str) -> str:
    return line.replace(",", " ").replace(";", " ")


def _read_blocks(path: str):
    """ConfigurationBase::extractArguments + extractRawContent (ConfigurationBase.cpp:57-121)."""
    try:
        with open(path, "r") as fh:
            lines = fh.read().split("\n")
    except OSError as exc:
        raise ValueError(f"ConfigurationBase: file does not exist: {path}") from exc
    # A trailing newline does not make an extra (empty) line.
    if lines and lines[-1] == "":
        lines = lines[:-1]
    found: List[str] = []
    contents: Dict[str, List[str]] = {}
    arg = ""
    content: List[str] = []
    for idx, line in enumerate(lines):
        if "#" in line:
            # extractArguments only records keys that are not on the last line
            if idx != len(lines) - 1:
                found.append(_parse_argument(line))
            if content:
                contents[arg] = content
                content = []
            arg = _parse_argument(line)
        elif not line or "!" in line:
            pass
        else:
            content.append(_standarize(line))
    contents[arg] = content
    return found, contents


def _floats(line: str) -> List[float]:
    return [float(t) for t in line.split()]


def _parse_number_prefix(tok: str) -> float:
    """istream >> double on a token: the longest numeric prefix ("+0.5j" -> 0.5)."""
    best = None
    for end in range(len(tok), 0, -1):
        try:
            best = float(tok[:end])
            break
        except ValueError:
            continue
    if best is None:
        raise ValueError(f"cannot parse number from {tok!r}")
    return best


def _parse_matrices(content: List[str]) -> np.ndarray:
    """SystemConfiguration::parseMatrices (SystemConfiguration.cpp:159-228).

    Returns an array [nmat][row][col] complex128."""
    first = content[0]
    is_complex = ("i" in first) or ("j" in first)
    ndim = 0
    for line in content:
        if "&" in line:
            break
        ndim += 1
    mats = []
    mat = np.zeros((ndim, ndim), dtype=np.complex128)
    row_index = 0
    for line in content:
        if "&" in line:
            mats.append(mat.copy())
            mat[:] = 0
            row_index = 0
            continue
        toks = line.split()
        row = np.zeros(ndim, dtype=np.complex128)
        j = 0
        t = 0
        while t < len(toks):
            re = _parse_number_prefix(toks[t])
            im = 0.0
            if is_complex:
                t += 1
                im = _parse_number_prefix(toks[t]) if t < len(toks) else 0.0
            row[j] = complex(re, im)
            j += 1
            t += 1
        mat[row_index] = row
        row_index += 1
    return np.array(mats, dtype=np.complex128).reshape(-1, ndim, ndim)


@dataclass
class SystemInfo:
    ndim: int = 0
    filling: float = 0.0
    bravaisLattice: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    motif: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    hamiltonian: np.ndarray = field(default_factory=lambda: np.zeros((0, 0, 0), dtype=np.complex128))
    overlap: np.ndarray = field(default_factory=lambda: np.zeros((0, 0, 0), dtype=np.complex128))
    bravaisVectors: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    norbitals: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))


class SystemConfiguration:
    """``.model`` reader (SystemConfiguration.cpp:20-258)."""

    expectedArguments = ["dimension", "bravaislattice", "motif", "norbitals", "filling", "bravaisvectors",
                         "hamiltonian"]

    def __init__(self, filename: str):
        if not filename:
            raise ValueError("ConfigurationBase: file must not be empty")
        self.filename = filename
        self.systemInfo = SystemInfo()
        self.foundArguments, self.contents = _read_blocks(filename)
        self._parse()
        for arg in self.expectedArguments:
            if arg not in self.foundArguments:
                raise ValueError("Missing arguments in config. file: missing " + arg)
        self._check()

    def _parse(self):
        info = self.systemInfo
        for arg in self.foundArguments:
            content = self.contents.get(arg, [])
            if arg == "dimension":
                if len(content) != 1:
                    raise ValueError("Expected only one line for 'Dimension'")
                info.ndim = int(_parse_number_prefix(content[0].split()[0]))
            elif arg == "bravaislattice":
                info.bravaisLattice = self._vectors(content)
            elif arg == "motif":
                rows = []
                for line in content:
                    vals = _floats(line)
                    if len(vals) < 4:
                        raise ValueError("Motif must be of shape (x,y,z,'species')")
                    rows.append(vals[:4])
                info.motif = np.array(rows, dtype=np.float64).reshape(-1, 4)
            elif arg == "norbitals":
                if len(content) != 1:
                    raise ValueError("Error: Orbital information must be one line only")
                info.norbitals = np.array([int(float(t)) for t in content[0].split()], dtype=np.int64)
            elif arg == "filling":
                if len(content) != 1:
                    raise ValueError("Expected only one line in 'filling' field")
                info.filling = float(content[0].split()[0])
                if info.filling != int(info.filling):
                    raise ValueError("Filling must be a positive integer.")
            elif arg == "bravaisvectors":
                info.bravaisVectors = self._vectors(content)
            elif arg == "hamiltonian":
                info.hamiltonian = _parse_matrices(content)
            elif arg == "overlap":
                info.overlap = _parse_matrices(content)

    @staticmethod
    def _vectors(content: List[str]) -> np.ndarray:
        out = []
        for line in content:
            v = _floats(line)
            if len(v) != 3:
                raise ValueError("Bravais vectors must have three components")
            out.append(v)
        return np.array(out, dtype=np.float64).reshape(-1, 3)

    def _check(self):
        """SystemConfiguration::checkContentCoherence (SystemConfiguration.cpp:235-258)."""
        info = self.systemInfo
        if info.ndim != info.bravaisLattice.shape[0]:
            raise ValueError("Error: Dimensions must match number of Bravais basis")
        if info.hamiltonian.shape[0] != info.bravaisVectors.shape[0]:
            raise ValueError("Error: Number of H matrices must match number of Bravais vectors")
        if info.overlap.size and info.overlap.shape[0] != info.hamiltonian.shape[0]:
            raise ValueError("Error: Number of overlap matrices must match number of H matrices")
        nspecies = len(set(int(s) for s in info.motif[:, 3]))
        if len(info.norbitals) != nspecies:
            raise ValueError("Error: Number of different species must match be consistent in motif and orbitals")


@dataclass
class ExcitonInfo:
    label: str = ""
    ncell: int = 0
    nbands: int = 0
    submeshFactor: int = 1
    bands: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    Q: np.ndarray = field(default_factory=lambda: np.zeros(3))
    shift: np.ndarray = field(default_factory=lambda: np.zeros(0))
    cutoff: float = 0.0
    eps: np.ndarray = field(default_factory=lambda: np.zeros(0))
    mode: str = "realspace"
    exchange: bool = False
    scissor: float = 0.0
    nReciprocalVectors: int = 0
    potential: str = "keldysh"
    exchangePotential: str = "keldysh"
    regularization: float = 0.0


class ExcitonConfiguration:
    """Exciton run-file reader (ExcitonConfiguration.cpp:21-156)."""

    supportedPotentials = ["keldysh", "coulomb"]

    def __init__(self, filename: str):
        self.filename = filename
        self.excitonInfo = ExcitonInfo()
        self.foundArguments, self.contents = _read_blocks(filename)
        self._parse()
        for arg in ("ncells", "dielectric"):
            if arg not in self.foundArguments:
                raise ValueError("Missing arguments in config. file: missing " + arg)
        self._check()

    def _parse(self):
        info = self.excitonInfo
        for arg in self.foundArguments:
            content = self.contents.get(arg, [])
            if len(content) == 0:
                continue
            if len(content) != 1:
                raise ValueError("Expected only one line per field")
            line = content[0]
            word = "".join(line.split()).lower()
            if arg == "label":
                info.label = line
            elif arg == "ncells":
                info.ncell = int(_parse_number_prefix(line.split()[0]))
            elif arg == "submesh":
                info.submeshFactor = int(_parse_number_prefix(line.split()[0]))
            elif arg == "shift":
                info.shift = np.array(_floats(line))
            elif arg == "bands":
                info.nbands = int(_parse_number_prefix(line.split()[0]))
            elif arg == "bandlist":
                info.bands = np.array([int(float(t)) for t in line.split()], dtype=np.int64)
            elif arg == "totalmomentum":
                info.Q = np.array(_floats(line))
            elif arg == "cutoff":
                info.cutoff = float(line.split()[0])
            elif arg == "dielectric":
                info.eps = np.array(_floats(line))
            elif arg == "reciprocal":
                info.mode = "reciprocalspace"
                info.nReciprocalVectors = int(_parse_number_prefix(line.split()[0]))
            elif arg == "exchange":
                if word not in ("true", "false"):
                    raise ValueError("Exchange option must be set to 'true' or 'false'.")
                info.exchange = word == "true"
            elif arg == "exchange.potential":
                info.exchangePotential = word
            elif arg == "potential":
                info.potential = word
            elif arg == "scissor":
                info.scissor = float(line.split()[0])
            elif arg == "regularization":
                info.regularization = float(line.split()[0])

    def _check(self):
        """ExcitonConfiguration::checkContentCoherence (ExcitonConfiguration.cpp:115-156)."""
        info = self.excitonInfo
        if info.Q.size != 3:
            raise ValueError("'Q' must be a 3d vector")
        if info.ncell <= 0:
            raise ValueError("'ncell' must be a positive number")
        if info.bands.size == 0 and info.nbands == 0:
            raise ValueError("'bands' must be specified")
        if info.eps.size == 0:
            raise ValueError("'dielectric' must be specified")
        if info.potential not in self.supportedPotentials:
            raise ValueError("Specified 'potential' not supported. Use 'keldysh' or 'coulomb'")
        if info.exchange and info.exchangePotential not in self.supportedPotentials:
            raise ValueError("Specified 'exchange.potential' not supported. Use 'keldysh' or 'coulomb'")
        if info.mode not in ("realspace", "reciprocalspace"):
            raise ValueError("Invalid mode. Use 'realspace' or 'reciprocalspace'")
