"""The FP64 reference gradient (reverse-mode autodiff of a torch restatement of
the path) against central finite differences (h = 1e-6, FP64) of the C/numpy
oracle: dE_n/dr0, dE_n/deps_m, dE_n/deps_s and directional derivatives along
Hermitian-consistent hopping perturbations, for the lowest exciton states.
Tolerance: 1e-5 relative to the gradient's scale."""
import numpy as np
import pytest

from grad_cases import CASES, PICKS, hopping_directions, oracle_case
from oracle.grad_reference import reference_gradients

NS = 3
H_FD = 1e-6


def _energies(case, HR=None, params=None):
    ex = oracle_case(case, HR=HR, params=params)
    return np.linalg.eigvalsh(ex.H)[:NS]


def test_struve_derivative_matches_fd():
    """d/dx of the reference's Struve approximation (autodiff) vs FD of the C restatement."""
    import torch
    from oracle.grad_reference import struve_h0
    from oracle.oracle import lib
    L = lib()
    for x in [0.01, 0.3, 2.0, 7.5, 12.0, 20.1, 35.0, 49.0, 60.0]:
        xt = torch.tensor([x], dtype=torch.float64, requires_grad=True)
        v = struve_h0(xt)
        (g,) = torch.autograd.grad(v.sum(), xt)
        assert abs(v.item() - L.orc_stvh0(x)) <= 1e-14 * max(1.0, abs(v.item()))
        h = 1e-6 * x
        fd = (L.orc_stvh0(x + h) - L.orc_stvh0(x - h)) / (2 * h)
        assert abs(g.item() - fd) <= 1e-6 * max(abs(fd), 1e-2), (x, g.item(), fd)


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_gradient_vs_fd(case):
    ex = oracle_case(case)
    ref = reference_gradients(ex, NS)
    np.testing.assert_allclose(ref["energies"], np.linalg.eigvalsh(ex.H)[:NS], rtol=0, atol=1e-9)
    p0 = list(CASES[case]["params"])
    # potential parameters: (eps_m, eps_s, r0) order of the parameters tuple
    for name, idx in [("eps_m", 0), ("eps_s", 1), ("r0", 2)]:
        h = H_FD * abs(p0[idx])
        pp, pm = list(p0), list(p0)
        pp[idx] += h
        pm[idx] -= h
        fd = (_energies(case, params=tuple(pp)) - _energies(case, params=tuple(pm))) / (2 * h)
        scale = max(np.abs(fd).max(), 1e-3)
        assert np.abs(ref[name] - fd).max() <= 1e-5 * scale, (name, ref[name], fd)
    # hoppings
    HR = np.array(ex.system.hamiltonian)
    G = ref["hamiltonian"]
    scale = np.abs(G).max(axis=(1, 2, 3))
    for d in hopping_directions(HR, ex.system.cells_h, PICKS):
        fd = (_energies(case, HR=HR + H_FD * d) - _energies(case, HR=HR - H_FD * d)) / (2 * H_FD)
        pred = np.array([np.real(np.sum(np.conj(G[n]) * d)) for n in range(NS)])
        assert np.all(np.abs(pred - fd) <= 1e-5 * scale), (pred, fd)
