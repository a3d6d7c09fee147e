"""The GPU engine against numbers the reference itself computed and saved
(decoded into tests/golden/ref_pins.npz from simulation/test_test_D2_X32/):

* the fg! energy of the reference's last optim_gs iterate (honeycomb XX,
  complex A (2,2,2,2,4), chi = 32): converge with the energy criterion, then
  the 4 iterations of run_gs and the energy, within 1e-10 of the saved value;
* effH and effN columns of the plaquette driver optim_es_h4 from the saved
  ground-state environment, tangent basis and plaquette MPO at two momenta,
  within 1e-7 (effH) and 1e-8 (effN) relative.
"""
import math
import os

import numpy as np
import pytest

import ipeps_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def pins():
    return np.load(os.path.join(GOLD, "ref_pins.npz"))


def test_gpu_reproduces_reference_gs_energy(engine, pkg):
    p = pins()
    H = [h.numpy() for h in O.honeycomb(1, 1, dir="XX")]
    cfg = pkg.default_config()
    x = p["gs_A"] / np.abs(p["gs_A"]).max()
    ts = pkg.CTMTensors(x, cfg, engine=engine)
    pkg.run_ctm(ts, conv_fun="energy", H=H)
    ts.Params["max_iter"] = ts.Params["ad_max_iter"]
    pkg.run_ctm(ts, conv_fun="energy", H=H)
    E, _ = pkg.get_gs_energy(ts, H)
    ts.close()
    assert abs(E.real - p["gs_energies"][-1]) <= 1e-10, (E.real, p["gs_energies"][-1])


@pytest.mark.parametrize("mom", [("0.1", "0"), ("1", "1")])
def test_gpu_reproduces_reference_effH_effN(engine, pkg, mom):
    """optim_es_h4 columns (get_es_grad_h4 with the saved plaquette MPO) from
    the saved environment: complex A, nested plaquette energy and its
    pullback w.r.t. B, get_all_norm."""
    p = pins()
    cfg = pkg.default_config()
    ts = pkg.CTMTensors(p["es_A"], cfg, engine=engine, init=False)
    C = [(p[f"es_C{k}"], p[f"es_E{k}"]) for k in range(1, 5)]
    for k in range(4):
        ts.set_CT(k + 1, *C[k])
    H4 = [p[f"es_H{k}"] for k in range(1, 5)]
    # the saved MPO is the subtracted Hamiltonian: zero plaquette energy
    assert abs(pkg.get_gs_energy_4x4(ts, H4)) <= 1e-12
    basis = p["es_basis"]
    refH, refN = p[f"effH_{mom[0]}_{mom[1]}"], p[f"effN_{mom[0]}_{mom[1]}"]
    for i in (0, 15, 30):
        colH, colN = pkg.drivers.es_column_h4(float(mom[0]), float(mom[1]), ts, H4, basis, i, C)
        eh = np.linalg.norm(colH - refH[:, i]) / np.linalg.norm(refH[:, i])
        en = np.linalg.norm(colN - refN[:, i]) / np.linalg.norm(refN[:, i])
        # effN (forward) 1e-8; effH goes through the nested pullback, which
        # amplifies the randomized projectors' 1e-10-level differences
        assert eh <= 1e-7 and en <= 1e-8, (mom, i, eh, en)
    ts.close()


def _wp_env(pkg, engine, p):
    ts = pkg.CTMTensors(p["wp_A"], pkg.default_config(), engine=engine, init=False)
    for k in range(1, 5):
        ts.set_CT(k, p[f"wp_C{k}"], p[f"wp_E{k}"])
    return ts


def _range_projector(X):
    Q, _ = np.linalg.qr(X)
    return Q @ Q.conj().T


def test_gpu_reproduces_reference_optim_wp(engine, pkg):
    """optim_wp (optim_wp.jl:133-193) on the device in the saved honeycomb
    environment with the XX plaquette operator (get_w_op): every effH/effN
    column the reference saved at site 1 (wp/HN.jld2) within 1e-10 relative,
    columns 1..10 of its site-2 run on the basis_1m sector (wp/HN_1m/1_10.jld2)
    likewise, and get_wp_basis on the device's effH/effN spanning the
    reference's sectors (projectors within 1e-8)."""
    p = pins()
    ts = _wp_env(pkg, engine, p)
    w = pkg.drivers.get_w_op()
    effH, effN = pkg.drivers.optim_wp(ts, w, p["wp_basis"], site=1)
    for i in range(effH.shape[1]):
        assert np.linalg.norm(effH[:, i] - p["wp_effH"][:, i]) <= 1e-10 * np.linalg.norm(p["wp_effH"][:, i]), i
        assert np.linalg.norm(effN[:, i] - p["wp_effN"][:, i]) <= 1e-10 * np.linalg.norm(p["wp_effN"][:, i]), i
    es, bp, bm = pkg.drivers.get_wp_basis(effH, effN, p["wp_basis"])
    assert bp.shape == p["wp_basis_1p"].shape and bm.shape == p["wp_basis_1m"].shape
    assert np.linalg.norm(_range_projector(bp) - _range_projector(p["wp_basis_1p"])) <= 1e-8
    assert np.linalg.norm(_range_projector(bm) - _range_projector(p["wp_basis_1m"])) <= 1e-8
    # the partial-save run: wp = 2, es_resume = 1, es_num = 10 on basis_1m
    h2, n2 = pkg.drivers.optim_wp(ts, w, p["wp_basis_1m"], site=2, es_resume=1, es_num=10)
    assert np.abs(h2[:, 10:]).max() == 0.0
    ref_h, ref_n = p["wp2_effH_1_10"], p["wp2_effN_1_10"]
    assert np.linalg.norm(h2[:, :10] - ref_h) <= 1e-10 * np.linalg.norm(ref_h)
    assert np.linalg.norm(n2[:, :10] - ref_n) <= 1e-10 * np.linalg.norm(ref_n)
    ts.close()


@pytest.mark.parametrize("site", [3, 4])
def test_gpu_wp_grad_matches_oracle_at_sites_3_and_4(engine, pkg, site):
    """get_wp_grad at the plaquette sites the reference's files do not cover,
    against the oracle's torch pullback (optim_wp.jl:195-220) with a random
    complex B: operator value and norm 1e-12, gH and gN 1e-10 relative."""
    import torch
    p = pins()
    ts = _wp_env(pkg, engine, p)
    rng = np.random.default_rng(site)
    B = rng.standard_normal(p["wp_A"].shape) + 1j * rng.standard_normal(p["wp_A"].shape)
    w = pkg.drivers.get_w_op()
    gH, gN, wv, nv = pkg.get_wp_grad(ts, pkg.drivers.get_local_h(w), B.reshape(-1, order="F"), site)
    T = torch.tensor
    tso = O.CTMTensors(A=T(p["wp_A"]), Ad=T(p["wp_A"].conj()), Cs=[T(p[f"wp_C{k}"]) for k in range(1, 5)],
                       Es=[T(p[f"wp_E{k}"]) for k in range(1, 5)], Params=dict(O.default_config()))
    oH, oN, ow, on = O.get_wp_grad(tso, O.get_w_op(), T(B.reshape(-1, order="F")), site)
    assert abs(wv - ow) <= 1e-12 * abs(ow) and abs(nv - on) <= 1e-12 * abs(on), (wv, ow, nv, on)
    assert np.linalg.norm(gH - oH.numpy()) <= 1e-10 * np.linalg.norm(oH.numpy())
    assert np.linalg.norm(gN - oN.numpy()) <= 1e-10 * np.linalg.norm(oN.numpy())
    ts.close()
