"""The oracle against numbers the reference itself computed and saved
(simulation/test_test_D2_X32/*.jld2, decoded into tests/golden/ref_pins.npz by
tests/golden/make_reference_pins.py).

* gs.jld2: the fg! energy of the reference's last optim_gs iterate (honeycomb
  XX model, complex A (2,2,2,2,4), default config chi = 32): reproduced to
  1e-12 (converge from init_ctm1 with the energy criterion, then the
  ad_max_iter = 4 iterations of run_gs and get_gs_energy, optim_gs.jl:53-91).
* es_{px}_{py}.jld2 (written by the plaquette driver optim_es_h4):
  effH = basis' * gH / 2 and effN = basis' * gN (optim_es_h4.jl:104-107) from
  the saved normalised ground-state environment, tangent basis and plaquette
  MPO: two columns at two momenta reproduced to 1e-9 relative.
"""
import importlib.util
import math
import os

import numpy as np
import pytest
import torch

import ipeps_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = "/root/reference/simulation/test_test_D2_X32"


def pins():
    return np.load(os.path.join(GOLD, "ref_pins.npz"))


def es_ts(p):
    cfg = O.default_config()
    T = torch.tensor
    return O.CTMTensors(A=T(p["es_A"]), Ad=T(p["es_A"].conj()), Cs=[T(p[f"es_C{k}"]) for k in range(1, 5)],
                        Es=[T(p[f"es_E{k}"]) for k in range(1, 5)], Params=dict(cfg))


def test_oracle_reproduces_reference_gs_energy():
    p = pins()
    H = O.honeycomb(1, 1, dir="XX")
    cfg = O.default_config()
    x = O.renormalize(torch.tensor(p["gs_A"]))
    with torch.no_grad():
        ts = O._detach_ts(O.get_conv_boundary(x, H, cfg))
        prm = dict(ts.Params)
        prm["max_iter"] = prm["ad_max_iter"]
        E = O.run_gs(ts.replace(Params=prm), H, x)
    assert abs(complex(E).real - p["gs_energies"][-1]) <= 1e-12, (complex(E).real, p["gs_energies"][-1])


def es_H(p):
    return [torch.tensor(p[f"es_H{k}"]) for k in range(1, 5)]


@pytest.mark.parametrize("mom", [("0.1", "0"), ("1", "1")])
def test_oracle_reproduces_reference_effH_effN(mom):
    """get_es_grad_h4 (optim_es_h4.jl:133-157) with the saved plaquette MPO:
    the nested CTMRG, the pullback w.r.t. B and get_all_norm."""
    p = pins()
    ts = es_ts(p)
    basis = p["es_basis"]
    H = es_H(p)
    prm = dict(ts.Params)
    prm.update(px=float(mom[0]) * math.pi, py=float(mom[1]) * math.pi)
    t1 = ts.replace(Params=prm)
    refH, refN = p[f"effH_{mom[0]}_{mom[1]}"], p[f"effN_{mom[0]}_{mom[1]}"]
    for i in (0, 30):
        gH, gN = O.get_es_grad_h4(t1, H, torch.tensor(basis[:, i]))
        colH = basis.conj().T @ gH.resolve_conj().numpy() / 2
        colN = basis.conj().T @ gN.resolve_conj().numpy()
        assert np.linalg.norm(colH - refH[:, i]) <= 1e-9 * np.linalg.norm(refH[:, i]), (mom, i)
        assert np.linalg.norm(colN - refN[:, i]) <= 1e-9 * np.linalg.norm(refN[:, i]), (mom, i)


def test_oracle_plaquette_energy_of_subtracted_hamiltonian_vanishes():
    """The saved MPO is get_local_h(h4 - E0 hI) (optim_es_h4.jl:170-183): its
    4x4 ground-state energy on the saved environment is 0."""
    p = pins()
    E = O.get_gs_energy_4x4(es_ts(p), es_H(p))
    assert abs(complex(E)) <= 1e-12


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_jld2_reader_matches_committed_pins(pkg):
    jld2 = pkg.jld2
    p = pins()
    gs = jld2.load(os.path.join(REF, "gs.jld2"))
    assert np.array_equal(gs["A"], p["gs_A"]) and np.array_equal(gs["energies"], p["gs_energies"])
    b = jld2.load(os.path.join(REF, "basis.jld2"))
    assert np.array_equal(b["basis"], p["es_basis"])
    assert [c.shape for c in b["ts"]["Cs"]] == [p[f"es_C{k}"].shape for k in range(1, 5)]
    e = jld2.load(os.path.join(REF, "es_1_1.jld2"))
    assert np.array_equal(e["effN"], p["effN_1_1"])
    # effN is Hermitian up to the columns' separate CTMRG convergence (rg_tol 1e-6)
    assert np.abs(e["effN"] - e["effN"].conj().T).max() <= 1e-6 * np.abs(e["effN"]).max()


def wp_ts(p):
    T = torch.tensor
    return O.CTMTensors(A=T(p["wp_A"]), Ad=T(p["wp_A"].conj()), Cs=[T(p[f"wp_C{k}"]) for k in range(1, 5)],
                        Es=[T(p[f"wp_E{k}"]) for k in range(1, 5)], Params=dict(O.default_config()))


@pytest.mark.parametrize("site,basis_key,effH_key,effN_key,cols", [
    (1, "wp_basis", "wp_effH", "wp_effN", [0, 31, 62]),
    (2, "wp_basis_1m", "wp2_effH_1_10", "wp2_effN_1_10", [0, 9]),
])
def test_oracle_reproduces_reference_optim_wp(site, basis_key, effH_key, effN_key, cols):
    """optim_wp (optim_wp.jl:133-193, get_wp_grad :195-220) with the honeycomb
    XX plaquette operator (get_w_op, honeycomb.jl:82-101) in the saved
    environment: the effH and effN columns the reference saved (wp/HN.jld2 at
    site 1, wp/HN_1m/1_10.jld2 at site 2 on the basis_1m sector), 1e-12 relative
    (measured ~1e-15)."""
    p = pins()
    ts = wp_ts(p)
    basis = torch.tensor(p[basis_key])
    out = O.optim_wp_columns(ts, O.get_w_op(), basis, cols, site=site)
    for (h, n), i in zip(out, cols):
        eh, en = p[effH_key][:, i], p[effN_key][:, i]
        assert np.linalg.norm(h.numpy() - eh) <= 1e-12 * np.linalg.norm(eh), (i, "effH")
        assert np.linalg.norm(n.numpy() - en) <= 1e-12 * np.linalg.norm(en), (i, "effN")


def _range_projector(X):
    Q, _ = np.linalg.qr(X)
    return Q @ Q.conj().T


def test_oracle_get_wp_basis_reproduces_reference_sectors():
    """get_wp_basis (optim_wp.jl:25-72) on the saved effH/effN: the positive and
    negative sectors span the reference's basis_1p and basis_1m (projectors
    within 1e-10; the eigenvectors themselves are defined up to normalisation)."""
    p = pins()
    es, bp, bm = O.get_wp_basis(torch.tensor(p["wp_effH"]), torch.tensor(p["wp_effN"]), torch.tensor(p["wp_basis"]))
    assert bp.shape == p["wp_basis_1p"].shape and bm.shape == p["wp_basis_1m"].shape
    assert np.linalg.norm(_range_projector(bp) - _range_projector(p["wp_basis_1p"])) <= 1e-10
    assert np.linalg.norm(_range_projector(bm) - _range_projector(p["wp_basis_1m"])) <= 1e-10
