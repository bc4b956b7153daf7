"""Band-window solve (eigenpairs of the band list only: Householder tridiagonalisation, Sturm multisection,
inverse iteration, one warp per k point) against the full Jacobi band solve and against H(k) of the oracle
system: energies to 1e-12 relative, eigenvectors of non-degenerate bands identical after the global phase
fix, residuals |H C - C E| and orthonormality of every returned column."""
import numpy as np
import pytest

from tests.helpers import engine_exciton, model_config, oracle_system
from xatu_b200.synthetic import random_honeycomb, synthetic_hexagonal

pytestmark = pytest.mark.gpu


def _stacks(cfg, ncell, nbands, params, backend, **kw):
    ex = engine_exciton(cfg, ncell, nbands, params, initialize=False, **kw)
    ex.setBandsBackend(backend)
    ex.initializeHamiltonian()
    out = ex.bandStacks()
    kp = ex.system.kpoints.copy()
    band_list = list(ex.valenceBands) + list(ex.conductionBands)
    ex.close()
    return out, kp, band_list


CASES = [
    ("hBN", lambda: model_config("hBN.model"), 12, 1, [1, 1, 10], {}),
    ("MoS2_Q", lambda: model_config("MoS2.model"), 9, 2, [1., 4., 13.55], {"Q": (0, 0.05, 0)}),
    ("syn22_4", lambda: synthetic_hexagonal(seed=1234), 12, 2, [1.0, 4.5, 40.0], {}),
    ("syn22_8", lambda: synthetic_hexagonal(seed=77), 10, 4, [1.0, 4.5, 40.0], {}),
    ("honey12_12", lambda: random_honeycomb(31, 12), 8, 6, [1.0, 3.0, 20.0], {}),
]


@pytest.mark.parametrize("name,make,ncell,nbands,params,kw", CASES, ids=[c[0] for c in CASES])
def test_window_matches_full_and_hamiltonian(name, make, ncell, nbands, params, kw):
    cfg = make()
    (evw, vvw, evqw, vvqw), kp, band_list = _stacks(cfg, ncell, nbands, params, "window", **kw)
    (evf, vvf, evqf, vvqf), _, _ = _stacks(cfg, ncell, nbands, params, "full", **kw)
    scale = max(1.0, np.abs(evf).max())
    assert np.abs(evw - evf).max() <= 1e-12 * scale
    assert np.abs(evqw - evqf).max() <= 1e-12 * scale
    sysr = oracle_system(cfg)
    Q = np.asarray(kw.get("Q", (0, 0, 0)), dtype=float)
    checked = 0
    for k in range(0, len(kp), max(1, len(kp) // 40)):
        for shift, ev, vw, vf in ((np.zeros(3), evw, vvw, vvf), (Q, evqw, vvqw, vvqf)):
            h = sysr.hamiltonian_k(kp[k] + shift)
            allw = np.linalg.eigvalsh(h)
            C = vw[k].T
            assert np.abs(h @ C - C * ev[k][None, :]).max() <= 1e-10 * scale
            assert np.abs(C.conj().T @ C - np.eye(C.shape[1])).max() <= 1e-11
            for b, rank in enumerate(band_list):
                gap = np.min(np.abs(np.delete(allw, rank) - allw[rank]))
                if gap > 1e-6 * scale:
                    assert np.abs(vw[k, b] - vf[k, b]).max() <= 1e-8, (name, k, b, gap)
                    checked += 1
    assert checked > 0
