"""CPU checks of the warm start's canonical gauge (ipeps.jl_b200/warmstart.py)
on an environment converged by the oracle.

* the boundaries: a random orthogonal matrix on each of the 4 boundary gauges,
  applied to both legs of the edge and to the two corner legs of the boundary,
  leaves the energy unchanged (a wrong pairing of legs would not);
* the canonical gauge: gauge_fix of the environment and of any such
  re-gauged copy give the same vector;
* the canonical form at full rank is an exact gauge transform (same energy),
  and unpack inverts the vector layout."""
import numpy as np
import torch

import ipeps_oracle as O
from conftest import load_package


def _converged(D=2, chi=6, seed=3):
    A = O.random_A(D, 2, seed=seed)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=40, rg_tol=1e-12)
    H = O.ising(2.0)
    ts = O.make_ctm_tensors(A, cfg)
    ts, _ = O.run_ctm(ts, conv_fun=lambda x: O.get_gs_energy(x, H)[0])
    return ts, H


def _energy(ts, Cs, Es, H):
    t = ts.replace(Cs=[torch.tensor(np.asarray(C)) for C in Cs], Es=[torch.tensor(np.asarray(E)) for E in Es])
    return complex(O.get_gs_energy(t, H)[0]).real


def test_bond_map_and_canonical_gauge():
    ws = load_package().warmstart
    ts, H = _converged()
    Cs = [c.numpy() for c in ts.Cs]
    Es = [e.numpy() for e in ts.Es]
    E0 = _energy(ts, Cs, Es, H)
    rng = np.random.default_rng(0)
    Qb = []
    for j in range(4):
        n = Es[j].shape[0]
        Qb.append(np.linalg.qr(rng.standard_normal((n, n)))[0])
    Cg, Eg = ws.gauge_transform(Cs, Es, Qb)
    assert abs(_energy(ts, Cg, Eg, H) - E0) <= 1e-12
    v = ws.gauge_fix(Cs, Es)
    vg = ws.gauge_fix(Cg, Eg)
    assert np.allclose(v, vg, atol=1e-10), np.abs(v - vg).max()
    r = Cs[0].shape[0]
    Cc, Ec = ws.unpack(v, r, Es[0].shape[2])
    assert abs(_energy(ts, Cc, Ec, H) - E0) <= 1e-12
    assert np.allclose(ws.gauge_fix(Cc, Ec), v, atol=1e-12)
