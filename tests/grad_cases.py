"""Systems of the gradient tests, shared by the CPU (reference gradient vs finite
differences of the oracle) and GPU (engine adjoint) test files."""
import numpy as np

from helpers import model_config, oracle_system
from oracle.oracle import OracleExciton, OracleSystem
from xatu_b200.synthetic import synthetic_hexagonal


def _syn(overlap=0.0):
    # 3 + 2 + 2 orbitals, full storage (H(-R) = H(R)^dagger), filling 3: bands 1..2 valence, 3..4 conduction
    return synthetic_hexagonal(seed=2024, orbitals=(3, 2, 2), a=3.0, sigma=0.5, onsite=2.0, shells=2,
                               overlap=overlap)


CASES = {
    "hbn_real": dict(model="hBN.model", ncell=6, nbands=1, params=(1.0, 5.0, 10.0)),
    "hbn_real_exch": dict(model="hBN.model", ncell=6, nbands=1, params=(1.0, 5.0, 10.0), exchange=True),
    "hbn_recip_exch": dict(model="hBN.model", ncell=6, nbands=1, params=(1.0, 5.0, 10.0), mode="reciprocalspace",
                           nG=3, exchange=True),
    "syn_real_exch": dict(model="syn", ncell=4, nbands=2, params=(1.0, 4.5, 40.0), exchange=True),
    "syn_Q": dict(model="syn", ncell=4, nbands=2, params=(1.0, 4.5, 40.0), Q=(0.05, 0.02, 0.0), exchange=True),
    "syn_overlap": dict(model="synS", ncell=4, nbands=2, params=(2.0, 3.0, 15.0)),
}


def config(case):
    m = CASES[case]["model"]
    if m == "syn":
        return _syn()
    if m == "synS":
        return _syn(overlap=0.08)
    return model_config(m)


def oracle_case(case, HR=None, params=None):
    """Initialised OracleExciton with its BSE matrix built (ex.H)."""
    c = CASES[case]
    cfg = config(case)
    base = oracle_system(cfg)
    s = base if HR is None else OracleSystem(base.ndim, base.bravais, base.motif, base.norbitals, base.cells_h,
                                             HR, base.filling, overlap=base.overlap, is_au=base.is_au)
    ex = OracleExciton(s, c["ncell"], c["nbands"], 0, params or c["params"], c.get("Q", (0, 0, 0)))
    ex.mode = c.get("mode", "realspace")
    ex.n_reciprocal = c.get("nG", 1)
    ex.exchange = c.get("exchange", False)
    ex.brillouin_zone_mesh(c["ncell"])
    ex.initialize_hamiltonian()
    ex.bs_hamiltonian()
    return ex


def engine_case(case):
    from xatu_b200.exciton import ExcitonTB
    c = CASES[case]
    ex = ExcitonTB(config(case), c["ncell"], c["nbands"], 0, c["params"], c.get("Q", (0, 0, 0)))
    ex.setMode(c.get("mode", "realspace"))
    ex.setReciprocalVectors(c.get("nG", 1))
    ex.setExchange(c.get("exchange", False))
    ex.brillouinZoneMesh(c["ncell"])
    ex.initializeHamiltonian()
    return ex


def hopping_directions(HR, cells, picks):
    """Hermitian-consistent perturbation directions dH of H(R): for each (r, a, b, phase) the entry
    H(R)_ab moves by phase and its partner H(-R)_ba by conj(phase)."""
    out = []
    for (r, a, b, ph) in picks:
        rm = int(np.argmin(np.linalg.norm(cells + cells[r], axis=1)))
        d = np.zeros_like(HR)
        d[r, a, b] += ph
        if not (r == rm and a == b):
            d[rm, b, a] += np.conj(ph)
        else:
            d[r, a, b] = ph.real   # a real diagonal entry of H(0)
        out.append(d)
    return out


PICKS = [(0, 0, 0, 1.0), (0, 0, 1, 1.0), (0, 0, 1, 1j), (1, 0, 1, 1.0), (1, 1, 0, 1j), (2, 1, 1, 0.6 + 0.8j)]
