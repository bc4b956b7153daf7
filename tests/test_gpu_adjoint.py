"""Adjoint (Hellmann-Feynman) gradients of the engine (xatu_adjoint):

* against the FP64 reference gradient (autodiff of the torch restatement, itself
  pinned to finite differences of the oracle in test_grad_reference.py);
* against central finite differences (h = 1e-6, FP64) of the engine's own FP64
  build + dense solve, on the 22-orbital model with 2v+2c bands;
* through a test-only torch.autograd.Function whose backward calls the adjoint,
  checked with torch.autograd.gradcheck.
"""
import numpy as np
import pytest
import torch

from grad_cases import CASES, PICKS, engine_case, hopping_directions, oracle_case
from oracle.grad_reference import reference_gradients
from xatu_b200 import _lib as L

pytestmark = pytest.mark.gpu

NS = 3


def _solve(ex, ns):
    ex.BShamiltonian("fp64")
    res = ex.diagonalize("diag", ns)
    return res.eigval[:ns], res.eigvec[:, :ns]


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_matches_reference_gradient(case):
    ex = engine_case(case)
    E, X = _solve(ex, NS)
    g = ex.adjointGradients(X)
    ref = reference_gradients(oracle_case(case), NS)
    np.testing.assert_allclose(E, ref["energies"], rtol=0, atol=1e-8)
    for n in range(NS):
        scale = np.abs(ref["hamiltonian"][n]).max()
        err = np.abs(g["hamiltonian"][n] - ref["hamiltonian"][n]).max()
        assert err <= 1e-8 * scale, (n, err, scale)
    for name in ("r0", "eps_m", "eps_s"):
        scale = max(np.abs(ref[name]).max(), 1e-6)
        assert np.abs(g[name] - ref[name]).max() <= 1e-8 * scale, (name, g[name], ref[name])
    ex.close()


def _syn22(ncell=8):
    from xatu_b200.exciton import ExcitonTB
    from xatu_b200.synthetic import synthetic_hexagonal
    cfg = synthetic_hexagonal(seed=1234)          # 8 + 7 + 7 = 22 orbitals
    ex = ExcitonTB(cfg, ncell, 2, 0, (1.0, 4.5, 40.0))
    ex.brillouinZoneMesh(ncell)
    ex.initializeHamiltonian()
    return ex


def test_adjoint_vs_engine_finite_differences_22_orbitals():
    """Lowest 4 energies of the 22-orbital model (2v + 2c), gradients w.r.t. r0, eps_m, eps_s and
    hopping directions vs central differences of the engine's FP64 path (h = 1e-6)."""
    ns = 4
    ex = _syn22()
    E0, X = _solve(ex, ns)
    g = ex.adjointGradients(X)
    h = 1e-6

    def energies():
        ex.initializeHamiltonian()
        return _solve(ex, ns)[0]

    p0 = (ex.eps_m, ex.eps_s, ex.r0)
    for name, idx in [("eps_m", 0), ("eps_s", 1), ("r0", 2)]:
        hh = h * abs(p0[idx])
        pp, pm = list(p0), list(p0)
        pp[idx] += hh
        pm[idx] -= hh
        ex.setParameters(pp)
        Ep = energies()
        ex.setParameters(pm)
        Em = energies()
        ex.setParameters(p0)
        fd = (Ep - Em) / (2 * hh)
        assert np.abs(g[name] - fd).max() <= 1e-5 * np.abs(fd).max(), (name, g[name], fd)
    HR = ex.system.hamiltonianMatrices.copy()
    scale = np.abs(g["hamiltonian"]).max(axis=(1, 2, 3))
    picks = PICKS + [(3, 5, 17, 1.0), (5, 21, 2, 1j), (0, 9, 9, 1.0)]
    for d in hopping_directions(HR, ex.system.unitCellList, picks):
        ex.system.hamiltonianMatrices = HR + h * d
        Ep = energies()
        ex.system.hamiltonianMatrices = HR - h * d
        Em = energies()
        fd = (Ep - Em) / (2 * h)
        pred = np.array([np.real(np.sum(np.conj(g["hamiltonian"][n]) * d)) for n in range(ns)])
        assert np.all(np.abs(pred - fd) <= 1e-5 * scale), (pred, fd)
    ex.system.hamiltonianMatrices = HR
    ex.close()


class EngineEnergies(torch.autograd.Function):
    """Test-only autograd wrapper: forward = the engine's FP64 build + dense solve (lowest ns energies),
    backward = xatu_adjoint."""

    @staticmethod
    def forward(ctx, HR, params, ex, ns):
        ex.system.hamiltonianMatrices = HR.detach().numpy().copy()
        ex.setParameters(params.detach().tolist())
        ex.initializeHamiltonian()
        E, X = _solve(ex, ns)
        g = ex.adjointGradients(X)
        P = np.stack([g["eps_m"], g["eps_s"], g["r0"]], axis=1)
        ctx.save_for_backward(torch.from_numpy(g["hamiltonian"]), torch.from_numpy(P))
        return torch.from_numpy(E.copy())

    @staticmethod
    def backward(ctx, gE):
        G, P = ctx.saved_tensors
        gH = torch.einsum("n,nrij->rij", gE.to(torch.complex128), G)
        gp = torch.einsum("n,np->p", gE, P)
        return gH, gp, None, None


def test_autograd_function_gradcheck():
    ex = engine_case("syn_real_exch")
    HR0 = torch.from_numpy(ex.system.hamiltonianMatrices.copy())
    cells = ex.system.unitCellList
    dirs = torch.from_numpy(np.stack(hopping_directions(ex.system.hamiltonianMatrices, cells, PICKS)))

    def f(t, params):
        HR = HR0 + torch.einsum("p,prij->rij", t.to(torch.complex128), dirs)
        return EngineEnergies.apply(HR, params, ex, NS)

    t = torch.zeros(len(PICKS), dtype=torch.float64, requires_grad=True)
    params = torch.tensor([1.0, 4.5, 40.0], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (t, params), eps=1e-6, atol=1e-6, rtol=1e-5)
    ex.close()


def test_adjoint_error_paths():
    ex = engine_case("hbn_real")
    E, X = _solve(ex, 2)
    with pytest.raises(L.XatuError):
        ex.adjointGradients(np.zeros((X.shape[0], 9), dtype=np.complex128))
    ev, vv, evq, vvq = ex.bandStacks()
    ex.upload_bands(ev, vv, evq, vvq)
    g = ex.adjointGradients(X, hamiltonian=False)       # potential gradients still defined
    assert np.all(np.isfinite(g["r0"]))
    with pytest.raises(L.XatuError):
        ex.adjointGradients(X)                           # hopping gradients need bands from the model
    ex.close()
