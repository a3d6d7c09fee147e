"""The host drivers above the engine on the GPU: optim_gs (L-BFGS with the
device E+grad unit), prepare_basis + optim_es + evaluate_es (one momentum).

* optim_gs: the same L-BFGS (drivers.optim_gs) run once with the device
  E+grad unit and once with the oracle's (energy_and_grad, CPU); the
  iterates agree to the E+grad parity level, so the energies after each step
  and the final energy agree to 1e-8.
* optim_es: band energies at (px, py) = (pi, 0) of a D=2 chi=8 Heisenberg
  state against the oracle's (tests/golden/es_d2.json: every basis vector's
  get_es_grad and evaluate_es on the CPU), 1e-6 absolute.  The tangent basis
  is a null space (not unique), so only basis-independent band energies are
  compared.
"""
import json
import os

import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_optim_gs_matches_oracle_lbfgs(engine, pkg):
    A0 = O.random_A(2, 2, seed=6).numpy()
    H = O.ising(2.0)
    Hn = [h.numpy() for h in H]
    cfg = pkg.default_config()
    cfg.update(chi=8, min_iter=4, max_iter=40, rg_tol=1e-10, ad_max_iter=4)

    def oracle_fg(A, H_, cfg_, engine=None):
        E, g, _ = O.energy_and_grad(torch.tensor(A), H, cfg_)
        return E, g.numpy(), None

    steps = 4
    r_gpu = pkg.drivers.optim_gs(Hn, A0, cfg, iterations=steps, engine=engine)
    r_ora = pkg.drivers.optim_gs(Hn, A0, cfg, iterations=steps, fg_fn=oracle_fg)
    assert len(r_gpu["energies"]) == len(r_ora["energies"]) >= 3
    assert np.allclose(r_gpu["energies"], r_ora["energies"], rtol=0, atol=1e-8), (r_gpu["energies"],
                                                                                  r_ora["energies"])
    # the optimisation lowers the energy
    assert r_gpu["energies"][-1] < r_gpu["energies"][0]


def test_optim_es_band_energies_match_oracle(engine, pkg):
    with open(os.path.join(GOLD, "es_d2.json")) as f:
        g = json.load(f)
    A = O.random_A(g["D"], g["d"], seed=g["seed"]).numpy()
    H = [h.numpy() for h in O.heisenberg(1.0)]
    cfg = pkg.default_config()
    cfg.update(chi=g["chi"], **g["cfg"])
    ts, H2, basis = pkg.drivers.prepare_basis(H, A, cfg, engine=engine)
    assert basis.shape == (A.size, A.size - 1)
    E0, _ = pkg.get_gs_energy(ts, H)
    assert abs(E0.real - g["E0"]) <= 1e-10
    effH, effN = pkg.drivers.optim_es(g["px"], g["py"], ts, H2, basis)
    es = pkg.drivers.band_energies(effH, effN, g["nrmB_cut"])
    eo = np.asarray(g["es"])
    assert len(es) == len(eo)
    assert np.allclose(es[:4], eo[:4], rtol=0, atol=1e-6), (es[:4], eo[:4])
    assert np.allclose(es, eo, rtol=1e-6, atol=1e-6)
    ts.close()


def test_optim_es_concurrent_contexts_match_oracle(engine, pkg):
    """optim_es with its basis vectors spread over three contexts (own streams,
    host threads) on one GPU: the same band energies as the oracle (1e-6)."""
    with open(os.path.join(GOLD, "es_d2.json")) as f:
        g = json.load(f)
    A = O.random_A(g["D"], g["d"], seed=g["seed"]).numpy()
    H = [h.numpy() for h in O.heisenberg(1.0)]
    cfg = pkg.default_config()
    cfg.update(chi=g["chi"], **g["cfg"])
    ts, H2, basis = pkg.drivers.prepare_basis(H, A, cfg, engine=engine)
    extra = [pkg.Engine(0), pkg.Engine(0)]
    try:
        effH, effN = pkg.drivers.optim_es(g["px"], g["py"], ts, H2, basis, engines=[engine] + extra)
    finally:
        for e in extra:
            e.close()
    assert np.all(np.abs(effN).sum(axis=0) > 0)  # every column computed
    es = pkg.drivers.band_energies(effH, effN, g["nrmB_cut"])
    eo = np.asarray(g["es"])
    assert len(es) == len(eo)
    assert np.allclose(es, eo, rtol=1e-6, atol=1e-6), (es[:4], eo[:4])
    ts.close()


@pytest.mark.parametrize("direction", ["h", "v"])
def test_correlation_TM_matches_oracle(engine, pkg, direction):
    """correlation_TM (expectation.jl:193-220): the leading transfer-matrix
    eigenvalue magnitudes of the converged environment, 1e-9 relative (the
    spectrum is gauge invariant)."""
    A = O.random_A(2, 2, seed=12)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=10, min_iter=4, max_iter=40, rg_tol=1e-11)
    ts_o = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts_o, _ = O.run_ctm(ts_o, conv_fun=lambda t: O.get_gs_energy(t, H)[0])
        eo, _ = O.correlation_TM(ts_o, direction, N=4)
    ts = pkg.CTMTensors(A.numpy(), cfg, engine=engine)
    pkg.run_ctm(ts, conv_fun="energy", H=[h.numpy() for h in H])
    es1, es, TM = pkg.drivers.correlation_TM(ts, direction, N=4)
    ts.close()
    eo = eo.numpy()
    assert np.allclose(es1[:4], eo[:4], rtol=1e-9), (es1[:4], eo[:4])


def test_correlation_TM_A_matches_oracle(engine, pkg):
    """correlation_TM_A (expectation.jl:185-191): CTMTensors(A, cfg), run_ctm
    with the spectrum criterion, correlation_TM; against the oracle's run_ctm
    (spectrum criterion) + correlation_TM, 1e-8 relative."""
    A = O.random_A(2, 2, seed=12)
    cfg = O.default_config()
    cfg.update(chi=10, min_iter=4, max_iter=60, rg_tol=1e-12)
    ts_o = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts_o, _ = O.run_ctm(ts_o)
        eo, _ = O.correlation_TM(ts_o, "h", N=4)
    es1, es, TM = pkg.drivers.correlation_TM_A(A.numpy(), cfg, direction="h", engine=engine)
    eo = eo.numpy()
    assert np.allclose(es1[:4], eo[:4], rtol=1e-8), (es1[:4], eo[:4])
