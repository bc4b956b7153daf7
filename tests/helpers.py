"""Shared helpers of the test-suite: fixtures paths, oracle set-up, engine runs."""
import json
import os

import numpy as np

from oracle.oracle import OracleExciton, OracleSystem
from xatu_b200.config import SystemConfiguration

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODELS = os.path.join(GOLDEN, "models")


def goldens():
    with open(os.path.join(GOLDEN, "reference_goldens.json")) as fh:
        return json.load(fh)


def model_config(name):
    return SystemConfiguration(os.path.join(MODELS, name))


def oracle_system(cfg):
    si = cfg.systemInfo
    ovl = si.overlap if getattr(si, "overlap", None) is not None and si.overlap.size else None
    return OracleSystem(si.ndim, si.bravaisLattice, si.motif, si.norbitals, si.bravaisVectors, si.hamiltonian,
                        int(si.filling), overlap=ovl)


def oracle_exciton(cfg, ncell, nbands, params, Q=(0, 0, 0), mode="realspace", nG=1, exchange=False, factor=None,
                   shift=None, cutoff=None, scissor=0.0, bands=None):
    ex = OracleExciton(oracle_system(cfg), ncell, nbands, 0, params, Q, bands=bands)
    ex.mode = mode
    ex.n_reciprocal = nG
    ex.exchange = exchange
    ex.scissor = scissor
    if cutoff is not None:
        ex.cutoff = cutoff
    if factor:
        ex.reduced_brillouin_zone_mesh(ncell, factor)
        ex.shift_bz(shift)
    else:
        ex.brillouin_zone_mesh(ncell)
    ex.initialize_hamiltonian()
    return ex


def engine_exciton(cfg, ncell, nbands, params, Q=(0, 0, 0), mode="realspace", nG=1, exchange=False, factor=None,
                   shift=None, cutoff=None, scissor=0.0, bands=None, initialize=True):
    from xatu_b200.exciton import ExcitonTB
    ex = ExcitonTB(cfg, ncell, nbands, 0, params, Q, bands=bands)
    ex.setMode(mode)
    ex.setReciprocalVectors(nG)
    ex.setExchange(exchange)
    ex.setScissor(scissor)
    if cutoff is not None:
        ex.setCutoff(cutoff)
    if factor:
        ex.system.reducedBrillouinZoneMesh(ncell, factor)
        ex.system.shiftBZ(shift)
    else:
        ex.brillouinZoneMesh(ncell)
    if initialize:
        ex.initializeHamiltonian()
    return ex


def case_kwargs(case):
    e = case["extra"]
    kw = {}
    if "mode" in e:
        kw["mode"] = e["mode"]
        kw["nG"] = e["nG"]
    if "Q" in e:
        kw["Q"] = tuple(e["Q"])
    if e.get("exchange"):
        kw["exchange"] = True
    if "factor" in e:
        kw["factor"] = e["factor"]
        kw["shift"] = e["shift"]
    return kw


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
