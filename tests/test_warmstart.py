"""CPU checks of the warm start's canonical gauge (ipeps.jl_b200/warmstart.py)
on an environment converged by the oracle.

* the boundaries: a random invertible matrix X on each of the 4 boundary
  gauges (E -> X^-1 E X, the facing corner legs absorbing X or X^-T) leaves the
  energy unchanged (a wrong pairing of corner and edge legs would not);
* the canonical gauge: gauge_fix of the environment and of a copy re-gauged by
  random orthogonal matrices give the same vector, and so do the environments
  after one and two more CTMRG iterations (CTMRG moves its fixed point only
  through orthogonal gauges, which gauge_fix removes);
* the canonical form at full rank is an exact gauge transform (same energy),
  and unpack inverts the vector layout."""
import numpy as np
import torch

import ipeps_oracle as O
from conftest import load_package


def _converged(D=2, chi=6, seed=3):
    A = O.random_A(D, 2, seed=seed)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=60, rg_tol=1e-13)
    H = O.ising(2.0)
    ts = O.make_ctm_tensors(A, cfg)
    ts, _ = O.run_ctm(ts, conv_fun=lambda x: O.get_gs_energy(x, H)[0])
    return ts, H


def _energy(ts, Cs, Es, H):
    t = ts.replace(Cs=[torch.tensor(np.asarray(C)) for C in Cs], Es=[torch.tensor(np.asarray(E)) for E in Es])
    return complex(O.get_gs_energy(t, H)[0]).real


def _env(ts):
    return [c.numpy() for c in ts.Cs], [e.numpy() for e in ts.Es]


def test_boundaries_and_canonical_gauge():
    ws = load_package().warmstart
    ts, H = _converged()
    Cs, Es = _env(ts)
    E0 = _energy(ts, Cs, Es, H)
    rng = np.random.default_rng(0)
    n = [E.shape[0] for E in Es]
    Xs = [np.eye(m) + 0.3 * rng.standard_normal((m, m)) for m in n]
    Cx, Ex = ws.gauge_transform(Cs, Es, Xs)
    assert abs(_energy(ts, Cx, Ex, H) - E0) <= 1e-12
    Qs = [np.linalg.qr(rng.standard_normal((m, m)))[0] for m in n]
    Cg, Eg = ws.gauge_transform(Cs, Es, Qs)
    assert abs(_energy(ts, Cg, Eg, H) - E0) <= 1e-12
    v = ws.gauge_fix(Cs, Es)
    vg = ws.gauge_fix(Cg, Eg)
    assert np.allclose(v, vg, atol=1e-10), np.abs(v - vg).max()
    r = Cs[0].shape[0]
    Cc, Ec = ws.unpack(v, r, Es[0].shape[2])
    assert abs(_energy(ts, Cc, Ec, H) - E0) <= 1e-12
    assert np.allclose(ws.gauge_fix(Cc, Ec), v, atol=1e-12)


def test_canonical_gauge_stable_under_ctmrg_iterations():
    ws = load_package().warmstart
    ts, H = _converged()
    v0 = ws.gauge_fix(*_env(ts))
    for _ in range(2):
        ts, _ = O.rg_step(ts, 6)
        v = ws.gauge_fix(*_env(ts))
        assert np.abs(v - v0).max() <= 1e-7, np.abs(v - v0).max()


def test_canonical_gauge_rectangular_corners():
    """A top boundary narrower than the others (as after a cutoff-limited
    truncation): corners C1, C2 are rectangular; the vector is zero-padded to
    rank r and still gauge invariant."""
    ws = load_package().warmstart
    ts, H = _converged()
    Cs, Es = _env(ts)
    rng = np.random.default_rng(5)
    W = np.linalg.qr(rng.standard_normal((Es[0].shape[0], 4)))[0]
    Cs[0], Cs[1] = Cs[0] @ W, W.T @ Cs[1]
    Es[0] = ws._apply_leg(ws._apply_leg(Es[0], 0, W), 1, W)
    n = [E.shape[0] for E in Es]
    assert n[0] == 4 and n[1] == 6
    v = ws.gauge_fix(Cs, Es, r=6)
    assert v.size == 4 * 36 + 4 * 36 * 4
    Qs = [np.linalg.qr(rng.standard_normal((m, m)))[0] for m in n]
    vg = ws.gauge_fix(*ws.gauge_transform(Cs, Es, Qs), r=6)
    assert np.allclose(v, vg, atol=1e-10), np.abs(v - vg).max()


def test_energy_bound():
    """The sanity bound a warm-started result must satisfy: |E| <= ||Hh|| + ||Hv||
    (Heisenberg S.S: 3/4 per bond); the oracle's converged energy lies inside."""
    ws = load_package().warmstart
    Hh = [h.numpy() for h in O.heisenberg(1.0)]
    assert abs(ws.energy_bound(Hh) - 1.5) < 1e-8
    ts, H = _converged()
    E = _energy(ts, *_env(ts), H)
    assert abs(E) <= ws.energy_bound([h.numpy() for h in H]) and 34.0 > ws.energy_bound([h.numpy() for h in H])
