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
* simulation/hb_test_D2_X32/ (test/optim_wp.jl): the honeycomb XX state's
  environment and tangent basis, effH/effN of optim_wp at plaquette site 1
  (wp/HN.jld2), the sectors of get_wp_basis (wp/basis_1m.jld2,
  wp/basis_1p.jld2) and columns 1..10 of the site-2 run (wp/HN_1m/1_10.jld2).

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
    # the plaquette-operator driver optim_wp (test/optim_wp.jl): honeycomb XX
    # ground state, its environment and tangent basis (basis.jld2), effH/effN of
    # the full basis at site 1 (wp/HN.jld2), the sectors get_wp_basis split it
    # into (wp/basis_1m.jld2, wp/basis_1p.jld2) and the columns 1..10 of the
    # site-2 run on basis_1m (wp/HN_1m/1_10.jld2)
    hb = os.path.join(ref_root, "simulation", "hb_test_D2_X32")
    hbb = jld2.load(os.path.join(hb, "basis.jld2"))
    hts = hbb["ts"]
    out["wp_A"] = hts["A"]
    out["wp_basis"] = hbb["basis"]
    for k in range(4):
        out[f"wp_C{k + 1}"] = hts["Cs"][k]
        out[f"wp_E{k + 1}"] = hts["Es"][k]
    hn = jld2.load(os.path.join(hb, "wp", "HN.jld2"))
    out["wp_effH"], out["wp_effN"] = hn["effH"], hn["effN"]
    out["wp_basis_1m"] = jld2.load(os.path.join(hb, "wp", "basis_1m.jld2"))["basis"]
    out["wp_basis_1p"] = jld2.load(os.path.join(hb, "wp", "basis_1p.jld2"))["basis"]
    hn1 = jld2.load(os.path.join(hb, "wp", "HN_1m", "1_10.jld2"))
    out["wp2_effH_1_10"], out["wp2_effN_1_10"] = hn1["effH"][:, :10], hn1["effN"][:, :10]
    np.savez_compressed(os.path.join(HERE, "ref_pins.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
