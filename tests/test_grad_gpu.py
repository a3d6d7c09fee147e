"""GPU energy + gradient (the pullback of run_gs inside fg!) against the
oracle's reference-adjoint gradient (torch autograd through the restated
moves with svd_back, autodiff.jl:41-74).

Bars (FP64 form): energy 1e-10 absolute; gradient 1e-6 relative (2-norm)."""
import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D,chi,model,seed", [(2, 8, "ising", 1), (2, 12, "heisenberg", 3), (3, 16, "heisenberg", 5)])
def test_energy_grad_matches_oracle(engine, pkg, D, chi, model, seed):
    A = O.random_A(D, 2, seed=seed)
    H = O.ising(2.0) if model == "ising" else O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, max_iter=40, min_iter=4, rg_tol=1e-11, ad_max_iter=4)
    Eo, go, _ = O.energy_and_grad(A, H, cfg)
    E, g, info = pkg.fg(A.numpy(), [h.numpy() for h in H], cfg, engine=engine)
    go = go.numpy()
    assert abs(E - Eo) <= 1e-10, (E, Eo)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel <= 1e-6, rel


def test_energy_grad_rectangular_environment(engine, pkg):
    """A near-product state (a product state plus 0.3 times Gaussian tensors,
    halfway along a straight path) whose cutoff-limited truncations leave
    boundaries of different bond dimensions (oracle: C1 16 x 14, C2 14 x 15,
    C3 15 x 16): the enlarged-corner matrices of the projector adjoint are
    rectangular (R1 N1 x K1, R2 K1 x N2 with N1, K1, N2 all different)."""
    rng = np.random.default_rng(3)
    prod = np.zeros((2, 2, 2, 2, 2))
    prod[0, 0, 0, 0, :] = rng.standard_normal(2)
    A0 = prod + 0.3 * rng.standard_normal(prod.shape)
    A1 = prod + 0.3 * rng.standard_normal(prod.shape)
    A = 0.5 * (A0 + A1)
    A = np.asfortranarray(A / np.abs(A).max())
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=16, max_iter=80, min_iter=4, rg_tol=1e-11, ad_max_iter=4)
    Eo, go, tso = O.energy_and_grad(torch.tensor(A), H, cfg)
    assert len({tuple(c.shape) for c in tso.Cs}) > 1
    E, g, info = pkg.fg(A, [h.numpy() for h in H], cfg, engine=engine)
    go = go.numpy()
    assert abs(E - Eo) <= 1e-10, (E, Eo)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel <= 1e-6, rel


def test_energy_grad_finite_difference(engine, pkg):
    """Directional derivatives of the GPU E+grad unit against central
    differences of the GPU energy of the same unit (step 1e-6)."""
    D, chi = 2, 8
    A = O.random_A(D, 2, seed=2).numpy()
    H = [h.numpy() for h in O.ising(2.0)]
    cfg = pkg.default_config()
    cfg.update(chi=chi, max_iter=40, min_iter=4, rg_tol=1e-12, ad_max_iter=4)
    x0 = A / np.abs(A).max()
    ts = pkg.CTMTensors(x0, cfg, engine=engine)
    ts, _ = pkg.run_ctm(ts, conv_fun="energy", H=H)
    C = [ts.get_CT(k) for k in range(1, 5)]
    E0, g = pkg.energy_grad(ts, H)

    def f(x):
        t = pkg.CTMTensors(x, cfg, engine=engine, init=False)
        for k in range(4):
            t.set_CT(k + 1, *C[k])
        e, _ = pkg.energy_grad(t, H)
        t.close()
        return e

    rng = np.random.default_rng(0)
    for _ in range(3):
        v = rng.standard_normal(A.shape)
        h = 1e-6
        fd = (f(x0 + h * v) - f(x0 - h * v)) / (2 * h)
        an = float((g * v).sum())
        # the reference adjoint broadens 1/(s_i^2 - s_j^2) (eta = 1e-12), so it is
        # not the exact derivative; agreement is at the 1e-4 level
        assert abs(fd - an) <= 1e-3 * abs(an) + 1e-7, (fd, an)


def test_es_grad_matches_oracle(engine, pkg):
    """Nested pullback w.r.t. B (get_es_grad, optim_es.jl:167-194): gH and gN
    against the oracle on a small ground-state environment (D=2, chi=8).
    Bars: gH and gN 1e-6 relative (2-norm)."""
    D, chi = 2, 8
    A = O.random_A(D, 2, seed=4)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=30, rg_tol=1e-10, ad_max_iter=4)
    ts_o = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts_o, _ = O.run_ctm(ts_o, conv_fun=lambda t: O.get_gs_energy(t, H)[0])
    ts_o = O._detach_ts(ts_o)
    g = np.random.default_rng(11)
    Bi = g.standard_normal(A.numel()) + 1j * g.standard_normal(A.numel())
    px, py = 0.5 * np.pi, 0.25 * np.pi
    ts_o.Params.update(px=px, py=py, max_iter=12, rg_tol=1e-8)
    gH_o, gN_o = O.get_es_grad(ts_o, H, torch.tensor(Bi))

    Hn = [h.numpy() for h in H]
    ts = pkg.CTMTensors(A.numpy(), cfg, engine=engine)
    pkg.run_ctm(ts, conv_fun="energy", H=Hn)
    ts.Params.update(px=px, py=py, max_iter=12, rg_tol=1e-8)
    gH, gN = pkg.get_es_grad(ts, Hn, Bi)
    gH_o, gN_o = gH_o.numpy(), gN_o.numpy()
    assert np.linalg.norm(gH - gH_o) <= 1e-6 * np.linalg.norm(gH_o), np.linalg.norm(gH - gH_o) / np.linalg.norm(gH_o)
    assert np.linalg.norm(gN - gN_o) <= 1e-6 * np.linalg.norm(gN_o)
