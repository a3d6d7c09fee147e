"""Generate tests/golden/ctm_energies.json from the CPU oracle.

The reference (Julia) cannot run in this environment, so the golden energies
of seeded synthetic cases come from the oracle, which is itself pinned to the
reference's honeycomb known-answer test.  Inputs are regenerated from seeds
(numpy default_rng, N(0,1), max|A| = 1, column-major).

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ipeps_oracle as O  # noqa: E402

CASES = [
    dict(model="ising", h=2.0, Jz=None, D=2, d=2, chi=16, seed=0, min_iter=4, max_iter=30, rg_tol=1e-10),
    dict(model="heisenberg", h=None, Jz=1.0, D=2, d=2, chi=12, seed=3, min_iter=4, max_iter=30, rg_tol=1e-10),
    dict(model="ising", h=2.0, Jz=None, D=2, d=2, chi=30, seed=0, min_iter=4, max_iter=30, rg_tol=1e-6),
    dict(model="heisenberg", h=None, Jz=1.0, D=3, d=2, chi=27, seed=1, min_iter=4, max_iter=30, rg_tol=1e-11),
]


def main():
    out = []
    for c in CASES:
        A = O.random_A(c["D"], c["d"], seed=c["seed"])
        H = O.ising(c["h"]) if c["model"] == "ising" else O.heisenberg(c["Jz"])
        cfg = O.default_config()
        cfg.update(chi=c["chi"], min_iter=c["min_iter"], max_iter=c["max_iter"], rg_tol=c["rg_tol"])
        log = []
        e0, _ = O.compute_gs_energy(A, H, cfg, log=log)
        c = dict(c)
        c["E"] = complex(e0).real
        c["iters"] = len(log)
        c["chi_final"] = log[-1]["chi"]
        out.append(c)
        print(c)
    with open(os.path.join(HERE, "ctm_energies.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py (CPU oracle, torch float64)", "cases": out}, f, indent=1)


def bench_workload(path=os.path.join(HERE, "bench_workload.json"), D=4, chi=64, iters=30, seed=1000):
    """Energy trajectory of a Heisenberg workload from init_ctm1 (default: D=4
    chi=64, seed 1000, 30 iterations; ~1 min of CPU).  The D=4 workload does
    not converge: it settles into a period-2 cycle, which makes it sensitive
    to the accuracy of the truncated SVD near the cut.  D=5 chi=100 with 8
    iterations (N = 2500 enlarged corners) takes several minutes."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    d = 2
    A = rng.standard_normal(D ** 4 * d).reshape((D, D, D, D, d), order="F")
    A = torch.tensor(np.asfortranarray(A / np.abs(A).max()))
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=iters, max_iter=iters, rg_tol=0.0)
    ts = O.make_ctm_tensors(A, cfg)
    traj = []
    for i in range(iters):
        ts, s = O.rg_step(ts, chi)
        traj.append(complex(O.get_gs_energy(ts, H)[0]).real)
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py:bench_workload (CPU oracle)", "model": "heisenberg",
                   "D": D, "d": d, "chi": chi, "seed": seed, "energies": traj}, f, indent=1)
    print("bench workload", traj[-2:])


def honeycomb_kat(path=os.path.join(HERE, "honeycomb_kat.json")):
    """The reference's energy known-answer cases (test/test_model.jl:9-16 and
    :78-83, -0.16349 +- 1e-5 for real(E)/8): complex A with d = 4, default
    config (chi = 32), converged from init_ctm1 with the energy criterion.
    Stores the oracle's energy trajectory and converged energy for each."""
    out = []
    for name, A, H in [("init_hb_gs_XX", O.init_hb_gs(2, p1=0.24, p2=0, dir="XX"), O.honeycomb(1, 1, dir="XX")),
                       ("ghz", O.get_Q_ghz(), O.honeycomb(1, 1))]:
        cfg = O.default_config()
        log = []
        E, Na = O.compute_gs_energy(A, H, cfg, log=log)
        E = complex(E)
        out.append({"name": name, "chi": cfg["chi"], "min_iter": cfg["min_iter"], "max_iter": cfg["max_iter"],
                    "rg_tol": cfg["rg_tol"], "E": [E.real, E.imag], "E_over_8": E.real / 8,
                    "iters": len(log), "trajectory": [complex(l["obj"]).real for l in log]})
        print(name, E.real / 8, len(log))
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py:honeycomb_kat (CPU oracle)", "cases": out}, f, indent=1)


if __name__ == "__main__":
    if "--bench-workload" in sys.argv:
        bench_workload()
    elif "--honeycomb" in sys.argv:
        honeycomb_kat()
    elif "--d5" in sys.argv:
        bench_workload(os.path.join(HERE, "d5_chi100.json"), D=5, chi=100, iters=8, seed=1000)
    else:
        main()
