"""The mixed form (3xTF32 contractions on the tensor cores, FP64 projector,
normalisation and energy, FP64 polish iterations at the end of a run) against
the FP64 oracle.

Bars: converged energy |dE| <= 1e-8 absolute; energy+gradient evaluation:
gradient 1e-6 relative (2-norm), energy 1e-8.
"""
import json
import os

import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def mixed_engine(pkg):
    eng = pkg.Engine(0, precision="mixed")
    yield eng
    eng.close()


def npa(t):
    return t.detach().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


@pytest.mark.parametrize("idx", [0, 1, 2, 3])
def test_mixed_converged_energy(mixed_engine, pkg, idx):
    with open(os.path.join(GOLD, "ctm_energies.json")) as f:
        case = json.load(f)["cases"][idx]
    A = npa(O.random_A(case["D"], case["d"], seed=case["seed"]))
    H = O.ising(case["h"]) if case["model"] == "ising" else O.heisenberg(case["Jz"])
    H = [npa(h) for h in H]
    cfg = O.default_config()
    cfg.update(chi=case["chi"], min_iter=case["min_iter"], max_iter=case["max_iter"], rg_tol=case["rg_tol"])
    (E, Na), ts, info = pkg.compute_gs_energy(A, H, cfg, engine=mixed_engine)
    if case["rg_tol"] <= 1e-10:
        # converged far below the bar: the fixed point itself
        assert abs(E.real - case["E"]) <= 1e-8, (E, case["E"])
    else:
        # rg_tol 1e-6: the energy depends on where the run stops, and the mixed
        # form stops after its FP64 polish iterations; against the FP64 form run
        # for the same number of iterations (pinned to the oracle elsewhere)
        c64 = dict(cfg)
        c64.update(min_iter=info["iters"], max_iter=info["iters"], rg_tol=0.0)
        (E64, _), t64, _ = pkg.compute_gs_energy(A, H, c64)
        t64.close()
        assert abs(E.real - E64.real) <= 1e-8, (E, E64)
    ts.close()


@pytest.mark.parametrize("D,chi,model,seed", [(2, 12, "heisenberg", 3), (3, 16, "heisenberg", 5)])
def test_mixed_energy_grad(mixed_engine, pkg, D, chi, model, seed):
    A = O.random_A(D, 2, seed=seed)
    H = O.ising(2.0) if model == "ising" else O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, max_iter=40, min_iter=4, rg_tol=1e-11, ad_max_iter=4)
    Eo, go, _ = O.energy_and_grad(A, H, cfg)
    E, g, info = pkg.fg(A.numpy(), [h.numpy() for h in H], cfg, engine=mixed_engine)
    go = go.numpy()
    assert abs(E - Eo) <= 1e-8, (E, Eo)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel <= 1e-6, rel
