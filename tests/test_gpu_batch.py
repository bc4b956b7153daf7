"""Batched build + solve (xatu_batch_*): every member's lowest energies against the
oracle (the CPU restatement of the reference: band solve, element loop, LAPACK
dense eigensolve) and against the single-system FP64 path (FP64 build + dense
eigensolve) of the same system, graph replays reproduce the first run, and the
autotuner reports a tile per class."""
import numpy as np
import pytest

from xatu_b200.batch import ExcitonBatch
from xatu_b200.synthetic import exciton_from_spec, random_honeycomb

pytestmark = pytest.mark.gpu

NST = 6


def _specs():
    rng = np.random.default_rng(77)
    out = []
    for i, (norb, ncell, nv, nc) in enumerate([(2, 8, 1, 1), (6, 10, 3, 3), (8, 12, 2, 3), (5, 9, 1, 2),
                                                (12, 8, 3, 1), (7, 11, 2, 2), (4, 10, 2, 2)]):
        cfg = random_honeycomb(900 + i, norb)
        out.append({"config": cfg, "ncell": ncell, "nv": nv, "nc": nc,
                    "params": (1.0, float(rng.uniform(1, 6)), float(rng.uniform(5, 50)))})
    return out


def _oracle(spec, nst, mode="realspace", nG=1, exchange=False):
    """Lowest nst energies of a batch member from the oracle (dense LAPACK solve of the oracle's H)."""
    from tests.helpers import oracle_exciton
    nv, nc = spec["nv"], spec["nc"]
    bands = list(range(-(nv - 1), 1)) + list(range(1, nc + 1))
    orc = oracle_exciton(spec["config"], spec["ncell"], 1, spec["params"], mode=mode, nG=nG, exchange=exchange,
                         bands=bands)
    return np.linalg.eigvalsh(orc.bs_hamiltonian())[:nst]


def _fp64(spec):
    ex = exciton_from_spec(spec)
    ex.initializeHamiltonian()
    ex.BShamiltonian("fp64")
    r = ex.diagonalize("diag", NST)
    ex.close()
    return r.eigval[:NST]


def test_batch_matches_single_system_fp64():
    specs = _specs()
    batch = ExcitonBatch()
    exs = [exciton_from_spec(s) for s in specs]
    for ex in exs:
        batch.add(ex)
    batch.run(NST)
    first = [batch.result(i)[0] for i in range(len(specs))]
    for i, s in enumerate(specs):
        ref = _fp64(s)
        assert np.abs(first[i] - ref).max() < 1e-4, (i, first[i], ref)
        orc = _oracle(s, NST)
        assert np.abs(first[i] - orc).max() < 1e-4, (i, first[i], orc)
    # eigenvectors come back normalised
    ev, vec = batch.result(1)
    assert np.allclose(np.linalg.norm(vec, axis=0), 1.0, atol=1e-10)
    # second run replays the recorded graphs (the floating-point atomics of the products and reductions
    # make runs differ in the last digits; the states are converged to residual 1e-4)
    batch.run(NST)
    for i in range(len(specs)):
        assert np.abs(batch.result(i)[0] - first[i]).max() < 1e-6
    st = batch.stats()
    assert st["iterations"] > 0 and st["solve_ms"] > 0 and st["build_ms"] > 0
    classes = {(c["nv"], c["nc"]) for c in st["tuning"]["assembly"]}
    assert classes == {(s["nv"], s["nc"]) for s in specs}
    assert all(c["chosen_tk"] in (8, 16) for c in st["tuning"]["assembly"])
    assert len(st["tuning"]["davidson"]) >= 1
    batch.close()
    for ex in exs:
        ex.close()


def test_batch_rejects_unsupported_member():
    batch = ExcitonBatch()
    spec = {"config": random_honeycomb(5, 2), "ncell": 4, "nv": 1, "nc": 1, "params": (1.0, 2.0, 10.0)}
    ex = exciton_from_spec(spec)        # N = 16 < basis size
    batch.add(ex)
    with pytest.raises(Exception):
        batch.run(NST)
    batch.close()
    ex.close()


def test_batch_exchange_and_reciprocal_members():
    """Members with the exchange term and in reciprocal-space mode, next to a plain one."""
    specs = _specs()[:3]
    settings = [dict(exchange=True), dict(mode="reciprocalspace", nG=3, exchange=True), dict()]

    def make(spec, opt):
        ex = exciton_from_spec(spec)
        ex.setExchange(opt.get("exchange", False))
        if "mode" in opt:
            ex.setMode(opt["mode"])
            ex.setReciprocalVectors(opt["nG"])
        return ex

    batch = ExcitonBatch()
    exs = [make(s, o) for s, o in zip(specs, settings)]
    for ex in exs:
        batch.add(ex)
    batch.run(NST)
    for i, (s, o) in enumerate(zip(specs, settings)):
        ref = make(s, o)
        ref.initializeHamiltonian()
        ref.BShamiltonian("fp64")
        e_ref = ref.diagonalize("diag", NST).eigval[:NST]
        ref.close()
        assert np.abs(batch.result(i)[0] - e_ref).max() < 1e-4, (i, o)
        e_orc = _oracle(s, NST, mode="reciprocalspace" if "mode" in o else "realspace", nG=o.get("nG", 1),
                        exchange=o.get("exchange", False))
        assert np.abs(batch.result(i)[0] - e_orc).max() < 1e-4, (i, o)
    batch.close()
    for ex in exs:
        ex.close()


def test_batch_restart_path_matches_fp64():
    """Members of the batched workload that need more lockstep steps than the basis holds (six blocks), so
    the thick restart (V <- U, W <- W Y, T <- diag(theta)) runs on the device; every member's lowest 8
    energies match the single-system FP64 build + dense solve."""
    from xatu_b200.synthetic import batch_workload
    specs = batch_workload(count=64)
    pick = [1, 13, 14, 38, 40, 46, 62]
    sub = [specs[i] for i in pick]
    batch = ExcitonBatch()
    exs = [exciton_from_spec(s) for s in sub]
    for ex in exs:
        batch.add(ex)
    batch.run(8)
    st = batch.stats()
    assert max(st["member_iterations"]) > 6, st["member_iterations"]
    for i, s in enumerate(sub):
        ex = exciton_from_spec(s)
        ex.initializeHamiltonian()
        ex.BShamiltonian("fp64")
        ref = ex.diagonalize("diag", 8).eigval[:8]
        ex.close()
        ev, vec = batch.result(i)
        assert np.abs(ev - ref).max() < 1e-4, (pick[i], ev, ref)
        assert np.allclose(np.linalg.norm(vec, axis=0), 1.0, atol=1e-10)
    batch.close()
    for ex in exs:
        ex.close()
