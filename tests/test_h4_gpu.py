"""Plaquette (4x4 cluster) observables of the engine against the oracle on a
real environment: get_gs_energy_4x4 and the nested get_es_energy_4x4, with
the MPO of a random Hermitian plaquette Hamiltonian (get_local_h), 1e-12
relative; the MPO reconstructs the Hamiltonian to rounding."""
import math

import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu


def _h4(seed, d=2):
    rng = np.random.default_rng(seed)
    n = d ** 4
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return ((X + X.conj().T) / 4).reshape(d * d, d * d, d * d, d * d, order="F")


def test_plaquette_energies_match_oracle(engine, pkg):
    A = O.random_A(2, 2, seed=9)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=12, min_iter=4, max_iter=30, rg_tol=1e-10)
    ts_o = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts_o, _ = O.run_ctm(ts_o, conv_fun=lambda t: O.get_gs_energy(t, H)[0])
    ts_o = O._detach_ts(ts_o)
    h = _h4(3)
    H4 = pkg.drivers.get_local_h(h)
    r = np.einsum("abx,xcdy,yefz,zgh->abcdefgh", *H4).reshape(h.shape, order="F")
    assert np.abs(r - h).max() <= 1e-13 * np.abs(h).max()
    H4t = [torch.tensor(x) for x in H4]
    Eo = complex(O.get_gs_energy_4x4(ts_o, H4t))
    ts = pkg.CTMTensors(A.numpy(), cfg, engine=engine, init=False)
    for k in range(4):
        ts.set_CT(k + 1, ts_o.Cs[k].numpy(), ts_o.Es[k].numpy())
    E = pkg.get_gs_energy_4x4(ts, H4)
    assert abs(E - Eo) <= 1e-12 * max(1.0, abs(Eo)), (E, Eo)
    # nested: B set, a few nested iterations with the plaquette criterion on both sides
    rng = np.random.default_rng(4)
    Bi = rng.standard_normal(A.numel()) + 1j * rng.standard_normal(A.numel())
    px, py = 0.5 * math.pi, 0.25 * math.pi
    prm = dict(ts_o.Params)
    prm.update(px=px, py=py)
    t1 = ts_o.replace(Params=prm, B=O.freshape(torch.tensor(Bi), *A.shape))
    t1 = t1.replace(Bd=O.conj(t1.B))
    Eeo = complex(O.get_es_energy_4x4(t1, H4t))
    ts.set_B(Bi.reshape(A.shape, order="F"), px, py)
    Ee = pkg.get_es_energy_4x4(ts, H4)
    assert abs(Ee - Eeo) <= 1e-12 * max(1.0, abs(Eeo)), (Ee, Eeo)
    ts.close()


def test_plaquette_energy_grad_matches_oracle(engine, pkg):
    """fg! of optim_gs_h4 (optim_gs_h4.jl:53-91): the plaquette energy and its
    gradient against the oracle's autograd, 1e-10 / 1e-6 relative."""
    A = O.random_A(2, 2, seed=13)
    h = _h4(5)
    H4 = pkg.drivers.get_local_h(h)
    cfg = O.default_config()
    cfg.update(chi=8, min_iter=4, max_iter=40, rg_tol=1e-11, ad_max_iter=4)
    Eo, go, _ = O.energy_and_grad_h4(A, [torch.tensor(x) for x in H4], cfg)
    E, g, info = pkg.host.fg_h4(A.numpy(), H4, cfg, engine=engine)
    go = go.numpy()
    assert abs(E - Eo) <= 1e-10 * max(1.0, abs(Eo)), (E, Eo)
    assert np.linalg.norm(g - go) <= 1e-6 * np.linalg.norm(go), np.linalg.norm(g - go) / np.linalg.norm(go)
