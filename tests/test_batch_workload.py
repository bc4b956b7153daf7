"""The batched workload's generator: seeded, sizes and ranges of the batched configuration
(random honeycomb models of 2-12 orbitals, k grids n x n with n in {24, 36, 48, 60}, 1-3 valence and
1-3 conduction bands within the model, r0 in [5, 50], eps_s in [1, 6], eps_m = 1)."""
import numpy as np

from xatu_b200.synthetic import batch_workload


def test_batch_workload_ranges_and_seed():
    w = batch_workload()
    assert len(w) == 64
    for s in w:
        info = s["config"].systemInfo
        norb = int(info.norbitals.sum())
        assert 2 <= norb <= 12
        assert s["ncell"] in (24, 36, 48, 60)
        n0 = int(info.filling)
        assert 1 <= s["nv"] <= min(3, n0) and 1 <= s["nc"] <= min(3, norb - n0)
        eps_m, eps_s, r0 = s["params"]
        assert eps_m == 1.0 and 1.0 <= eps_s <= 6.0 and 5.0 <= r0 <= 50.0
        H = info.hamiltonian
        # H(-R) = H(R)^dagger stored explicitly, Hermitian R = 0 block
        assert np.allclose(H[0], H[0].conj().T)
    w2 = batch_workload()
    assert all(a["ncell"] == b["ncell"] and a["params"] == b["params"] for a, b in zip(w, w2))
    assert np.allclose(w[5]["config"].systemInfo.hamiltonian, w2[5]["config"].systemInfo.hamiltonian)
