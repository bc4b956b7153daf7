"""Summed oscillator strength in an energy window (xatu_oscillator_window_gradient): the value against the
oracle (ResultTB::excitonOscillatorStrength restated, summed over the window) and dF/dr0, dF/deps_m,
dF/deps_s against central finite differences (h = 1e-6, FP64) of the oracle.  The window's upper edge is
placed in the middle of a spectral gap so that no state crosses it under the finite-difference steps."""
import numpy as np
import pytest

from grad_cases import CASES, engine_case, oracle_case
from oracle.oracle import exciton_oscillator_strength

pytestmark = pytest.mark.gpu

OSC_CASES = ["hbn_real", "hbn_real_exch", "hbn_recip_exch", "syn_real_exch"]


def _window(E, width=0.2):
    lo = E[0] - 1e-3
    k = int(np.searchsorted(E, E[0] + width, side="right")) - 1
    while k + 1 < len(E) and E[k + 1] - E[k] < 1e-3:
        k += 1
    hi = 0.5 * (E[k] + E[k + 1]) if k + 1 < len(E) else E[-1] + 1.0
    return lo, hi


def _oracle_F(case, lo, hi, params=None):
    ex = oracle_case(case, params=params)
    w, X = np.linalg.eigh(ex.H)
    sel = (w >= lo) & (w <= hi)
    v = exciton_oscillator_strength(ex, X[:, sel])
    return float(np.sum(np.abs(v) ** 2)), int(sel.sum())


@pytest.mark.parametrize("case", OSC_CASES)
def test_oscillator_window_value_and_gradient(case):
    ex = engine_case(case)
    ex.BShamiltonian("fp64")
    E = ex.diagonalize("diag", 1).eigval
    lo, hi = _window(np.sort(E))
    g = ex.oscillatorWindowGradient(lo, hi)
    ex.close()
    F0, nw = _oracle_F(case, lo, hi)
    assert g["nwindow"] == nw and nw >= 1
    assert abs(g["F"] - F0) <= 1e-8 * max(F0, 1e-12)
    p0 = list(CASES[case]["params"])
    for name, idx in [("eps_m", 0), ("eps_s", 1), ("r0", 2)]:
        h = 1e-6 * abs(p0[idx])
        pp, pm = list(p0), list(p0)
        pp[idx] += h
        pm[idx] -= h
        Fp, nwp = _oracle_F(case, lo, hi, tuple(pp))
        Fm, nwm = _oracle_F(case, lo, hi, tuple(pm))
        assert nwp == nw and nwm == nw
        fd = (Fp - Fm) / (2 * h)
        assert abs(g[name] - fd) <= 1e-5 * max(abs(fd), 1e-6 * F0), (name, g[name], fd)


def _oracle_F_hr(case, lo, hi, HR):
    ex = oracle_case(case, HR=HR)
    w, X = np.linalg.eigh(ex.H)
    sel = (w >= lo) & (w <= hi)
    v = exciton_oscillator_strength(ex, X[:, sel])
    return float(np.sum(np.abs(v) ** 2)), int(sel.sum())


@pytest.mark.parametrize("case", ["hbn_real", "hbn_recip_exch", "syn_real_exch"])
def test_oscillator_window_hopping_gradient(case):
    """dF/dH(R) through the eigenvectors, the bands and the velocity matrix elements, against central
    differences of the oracle along Hermitian-consistent hopping directions."""
    from grad_cases import PICKS, hopping_directions
    ex = engine_case(case)
    ex.BShamiltonian("fp64")
    E = ex.diagonalize("diag", 1).eigval
    lo, hi = _window(np.sort(E))
    g = ex.oscillatorWindowGradient(lo, hi, gradient=False, hamiltonian=True)
    HR = ex.system.hamiltonianMatrices.copy()
    cells = ex.system.unitCellList
    ex.close()
    G = g["hamiltonian"]
    scale = np.abs(G).max()
    h = 1e-6
    for d in hopping_directions(HR, cells, PICKS):
        Fp, nwp = _oracle_F_hr(case, lo, hi, HR + h * d)
        Fm, nwm = _oracle_F_hr(case, lo, hi, HR - h * d)
        assert nwp == g["nwindow"] and nwm == g["nwindow"]
        fd = (Fp - Fm) / (2 * h)
        pred = float(np.real(np.sum(np.conj(G) * d)))
        assert abs(pred - fd) <= 1e-5 * scale, (pred, fd, scale)
