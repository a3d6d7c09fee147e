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
