"""The GPU engine against numbers the reference itself computed and saved
(decoded into tests/golden/ref_pins.npz from simulation/test_test_D2_X32/):

* the fg! energy of the reference's last optim_gs iterate (honeycomb XX,
  complex A (2,2,2,2,4), chi = 32): converge with the energy criterion, then
  the 4 iterations of run_gs and the energy, within 1e-10 of the saved value;
* effN columns of optim_es from the saved ground-state environment and
  tangent basis at two momenta, within 1e-8 relative.
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
def test_gpu_reproduces_reference_effN(engine, pkg, mom):
    p = pins()
    cfg = pkg.default_config()
    A = p["es_A"]
    ts = pkg.CTMTensors(A, cfg, engine=engine, init=False)
    C = [(p[f"es_C{k}"], p[f"es_E{k}"]) for k in range(1, 5)]
    for k in range(4):
        ts.set_CT(k + 1, *C[k])
    H2 = pkg.drivers.substract_gs_energy(ts, [h.numpy() for h in O.ising(2.0)])
    basis = p["es_basis"]
    ref = p[f"effN_{mom[0]}_{mom[1]}"]
    for i in (0, 15, 30):
        _, colN = pkg.drivers.es_column(float(mom[0]), float(mom[1]), ts, H2, basis, i, C)
        assert np.linalg.norm(colN - ref[:, i]) <= 1e-8 * np.linalg.norm(ref[:, i]), (
            mom, i, np.linalg.norm(colN - ref[:, i]) / np.linalg.norm(ref[:, i]))
    ts.close()
