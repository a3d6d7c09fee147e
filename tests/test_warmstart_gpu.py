"""The learned warm start on the device: the network (BF16 tensor-core GEMMs)
is trained on canonical-gauge environments converged by plain CTMRG along
straight paths through the space of D=2 iPEPS tensors, then predicts the
starting environment for held-out points of the same paths.

Bars: the warm-started run reaches the same energy as plain CTMRG from
init_ctm1 (|dE| <= 1e-8 at rg_tol 1e-10) and every held-out start converges
without the fallback; a warm start given too few iterations falls back to
init_ctm1 and returns exactly the plain-CTMRG energy.  The iteration counts of
both starts are reported, not asserted: how many iterations a start saves
depends on the states (near a slow fixed point even the exact environment of a
neighbouring point saves only a few)."""
import numpy as np
import pytest

import ipeps_oracle as O

pytestmark = pytest.mark.gpu

D, d, CHI, R = 2, 2, 16, 16


def _cfg(**kw):
    cfg = O.default_config()
    cfg.update(chi=CHI, min_iter=4, max_iter=200, rg_tol=1e-10)
    cfg.update(kw)
    return cfg


@pytest.fixture(scope="module")
def trained(pkg, engine):
    ws_mod = pkg.warmstart
    H = [h.numpy() for h in O.heisenberg(1.0)]
    fam = ws_mod.path_family(D, d, seeds=range(4), n_points=9)
    train = [x for i, x in enumerate(fam) if i % 9 % 2 == 0]
    held = [x for i, x in enumerate(fam) if i % 9 % 2 == 1]
    targets = []
    for _, _, A in train:
        ts, info = ws_mod.converge_default(A, H, _cfg(), engine=engine)
        assert info["converged"]
        targets.append(ws_mod.gauge_fix(*ws_mod.read_env(ts), r=R))
        ts.close()
    ws = ws_mod.WarmStart(D, d, r=R, hidden=256, max_batch=64, seed=1, engine=engine)
    losses = ws.fit([A for _, _, A in train], np.stack(targets), epochs=800, lr=1e-3)
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])
    yield ws, H, held
    ws.close()


def test_warm_start_matches_plain_ctmrg(pkg, engine, trained):
    ws, H, held = trained
    res = pkg.warmstart.evaluate([A for _, _, A in held[::2]], H, _cfg(), ws, engine=engine)
    assert res["max_dE"] <= 1e-8, res["max_dE"]
    assert res["warm_used"] == res["n"], [r["used_warm"] for r in res["rows"]]
    print("iterations: default %.2f, warm start %.2f" % (res["mean_iters_default"], res["mean_iters_warm"]))


def test_warm_start_fallback(pkg, engine, trained):
    ws, H, held = trained
    A = held[1][2]
    ts0, _ = pkg.warmstart.converge_default(A, H, _cfg(), engine=engine)
    E0 = pkg.get_gs_energy(ts0, H)[0].real
    ts0.close()
    ts, info, used, iters = ws.converge(A, H, _cfg(), warm_max_iter=2)
    assert not used and info["converged"]
    assert abs(pkg.get_gs_energy(ts, H)[0].real - E0) <= 1e-12  # the same run from init_ctm1
    ts.close()
