"""Decode the reference's own saved results (its simulation/*.jld2 files) into
committed fixtures: tests/golden/ref_pins.npz.

iPEPS.jl ships the outputs of its test scripts (test/optim_gs.jl,
test/optim_es.jl) under simulation/test_test_D2_X32/.  Two of them pin the
oracle, and through it the GPU engine, to numbers the reference itself
computed:

* gs.jld2 (the last optim_gs run of test/optim_gs.jl: honeycomb XX model,
  complex A of shape (2,2,2,2,4), default config chi=32): the optimised A and
  the energy of fg! at it (energies[end]).
* basis.jld2 + es_{px}_{py}.jld2 (the plaquette excited-state driver,
  optim_es_h4.jl, D=2 d=2): the normalised ground state with its converged
  environment (ts.A, ts.Cs, ts.Es), the tangent basis, the plaquette
  Hamiltonian with E0 subtracted as the MPO list [s1, s2, s3, s4] of
  get_local_h (basis.jld2 "H"), and effH = basis' * gH / 2,
  effN = basis' * gN per momentum (optim_es_h4.jl:104-107).

Usage (reads the reference tree, so it runs where that tree is):
    python tests/golden/make_reference_pins.py /path/to/iPEPS.jl
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
spec = importlib.util.spec_from_file_location("jld2", os.path.join(HERE, "..", "..", "ipeps.jl_b200", "jld2.py"))
jld2 = importlib.util.module_from_spec(spec)
spec.loader.exec_module(jld2)

MOMENTA = [("0.1", "0"), ("1", "1"), ("0.5", "0.5")]


def main(ref_root):
    sim = os.path.join(ref_root, "simulation", "test_test_D2_X32")
    gs = jld2.load(os.path.join(sim, "gs.jld2"))
    b = jld2.load(os.path.join(sim, "basis.jld2"))
    ts = b["ts"]
    out = {
        "gs_A": gs["A"], "gs_energies": gs["energies"],
        "es_A": ts["A"], "es_basis": b["basis"],
    }
    for k in range(4):
        out[f"es_C{k + 1}"] = ts["Cs"][k]
        out[f"es_E{k + 1}"] = ts["Es"][k]
    for k in range(4):
        out[f"es_H{k + 1}"] = b["H"][k]
    for px, py in MOMENTA:
        e = jld2.load(os.path.join(sim, f"es_{px}_{py}.jld2"))
        out[f"effN_{px}_{py}"] = e["effN"]
        out[f"effH_{px}_{py}"] = e["effH"]
    np.savez_compressed(os.path.join(HERE, "ref_pins.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
