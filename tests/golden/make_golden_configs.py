"""Golden fixtures of the benchmark configurations, from the CPU oracle.

The reference (Julia) cannot run here, so these come from the oracle
restatement (torch float64 / complex128), which the CPU tests pin to the
reference's own known answers.  Inputs are regenerated from seeds (numpy
default_rng, N(0,1), max|A| = 1, column-major).

    python tests/golden/make_golden_configs.py config1   # TFIM D=2 chi=30, spectrum criterion + E+grad
    python tests/golden/make_golden_configs.py config2   # Heisenberg D=4 chi=64, 30 iterations: E, spectrum, grad
    python tests/golden/make_golden_configs.py config5   # Heisenberg D=3 chi=48: get_es_grad of 3 basis vectors
    python tests/golden/make_golden_configs.py d5        # Heisenberg D=5 chi=100, 30 iterations: energies
    python tests/golden/make_golden_configs.py es_d2     # Heisenberg D=2 chi=8: band energies at (pi, 0)

Each writes tests/golden/<name>.json.  Complex vectors are stored as
[re, im] pairs; tensors flattened in column-major (Julia) order.
"""
import json
import math
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ipeps_oracle as O  # noqa: E402


def flat(t):
    """column-major flattening of a real tensor"""
    return np.asarray(O.freshape(t.detach(), -1).resolve_conj().numpy(), dtype=np.float64).tolist()


def cflat(t):
    v = O.freshape(t.detach(), -1).resolve_conj().numpy()
    return [[float(z.real), float(z.imag)] for z in v]


def dump(name, obj):
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(obj, f)
    print("wrote", name)


def _spectrum_run(A, H, cfg):
    """run_ctm without conv_fun (spectrum criterion, ctmrg.jl:29-31) from init_ctm1."""
    log = []
    ts = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts, conv = O.run_ctm(ts, conv_fun=None, log=log)
    return O._detach_ts(ts), conv, log


def _grad_from(ts, H, x):
    """the pullback half of fg! (optim_gs.jl:62-80) from the converged env ts"""
    p = dict(ts.Params)
    p["max_iter"] = p.get("ad_max_iter", 4)
    ts = ts.replace(Params=p)
    xv = x.clone().requires_grad_(True)
    y = O.run_gs(ts, H, xv)
    yr = y.real if torch.is_complex(y) else y
    (g,) = torch.autograd.grad(yr, xv)
    return float(yr.item()), g.detach()


def config1():
    """TFIM h=2, A (2,2,2,2,2) seed 0, chi=30, min_iter 4, max_iter 30,
    rg_tol 1e-6 on the corner spectrum; then energy and gradient (pullback
    of ad_max_iter = 4 iterations).  Also the fg! path (energy criterion)."""
    A = O.random_A(2, 2, seed=0)
    H = O.ising(2.0)
    cfg = O.default_config()
    cfg.update(chi=30, min_iter=4, max_iter=30, rg_tol=1e-6, ad_max_iter=4)
    ts, conv, log = _spectrum_run(A, H, cfg)
    E_conv = float(complex(O.get_gs_energy(ts, H)[0]).real)
    E, g = _grad_from(ts, H, A)
    Ef, gf, tsf = O.energy_and_grad(A, H, cfg)
    dump("config1", {
        "generator": "tests/golden/make_golden_configs.py config1 (CPU oracle)",
        "model": "ising", "h": 2.0, "D": 2, "d": 2, "chi": 30, "seed": 0, "min_iter": 4, "max_iter": 30,
        "rg_tol": 1e-6, "ad_max_iter": 4,
        "spectrum": {"iters": len(log), "diffs": [float(l["diff"]) for l in log],
                     "s_last": [float(x) for x in conv.numpy()], "E_converged": E_conv,
                     "E_ad": E, "grad": flat(g)},
        "energy_criterion": {"E": Ef, "grad": flat(gf)},
    })


def config2(iters=30, seed=1000, ndir=16):
    """Heisenberg D=4 chi=64, seed 1000, 30 iterations from init_ctm1 (no
    early stop): energies per iteration, the left-move spectrum of the last
    iteration, then E+grad (pullback of 4 iterations) and the directional
    derivatives along 16 seeded directions."""
    A = O.random_A(4, 2, seed=seed)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=64, min_iter=iters, max_iter=iters, rg_tol=0.0, ad_max_iter=4)
    t0 = time.time()
    ts = O.make_ctm_tensors(A, cfg)
    traj = []
    with torch.no_grad():
        for _ in range(iters):
            ts, s = O.rg_step(ts, 64)
            traj.append(float(complex(O.get_gs_energy(ts, H)[0]).real))
    ts = O._detach_ts(ts)
    print("config2 forward", time.time() - t0)
    E, g = _grad_from(ts, H, A)
    print("config2 grad", time.time() - t0)
    rng = np.random.default_rng(77)
    dirs = rng.standard_normal((ndir, A.numel()))
    gflat = np.asarray(flat(g))
    dump("config2", {
        "generator": "tests/golden/make_golden_configs.py config2 (CPU oracle)",
        "model": "heisenberg", "D": 4, "d": 2, "chi": 64, "seed": seed, "iters": iters, "ad_max_iter": 4,
        "energies": traj, "s_last": [float(x) for x in s.numpy()], "E_ad": E, "grad": gflat.tolist(),
        "direction_seed": 77, "directional": (dirs @ gflat).tolist(),
    })


def config5(seed=21, chi=48, vec_cols=(0, 80, 160)):
    """Heisenberg D=3 chi=48, A seeded: converge the ground-state environment
    (energy criterion), normalise A, subtract E0/2 from H (prepare_basis,
    optim_es.jl:34-73), take the default tangent basis, and get_es_grad of
    three basis vectors at (px, py) = (pi, 0) and (pi/2, pi/2)."""
    A = O.random_A(3, 2, seed=seed)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=40, rg_tol=1e-10, ad_max_iter=4)
    t0 = time.time()
    ts = O.make_ctm_tensors(A, cfg)
    with torch.no_grad():
        ts, _ = O.run_ctm(ts, conv_fun=lambda t: O.get_gs_energy(t, H)[0])
        ts = O._detach_ts(ts)
        ts = O.normalize_gs(ts)
        H2 = O.substract_gs_energy(ts, H)
        basis = O.get_tangent_basis(ts)
    print("config5 gs", time.time() - t0)
    out = []
    for px, py in [(math.pi, 0.0), (0.5 * math.pi, 0.5 * math.pi)]:
        for col in vec_cols:
            Bi = basis[:, col]
            p = dict(ts.Params)
            p.update(px=px, py=py, max_iter=20, min_iter=4, rg_tol=1e-8)
            t1 = ts.replace(Params=p)
            gH, gN = O.get_es_grad(t1, H2, Bi)
            out.append({"px": px, "py": py, "col": col, "Bi": cflat(Bi), "gH": cflat(gH), "gN": cflat(gN)})
            print("config5", px, py, col, time.time() - t0)
    dump("config5", {
        "generator": "tests/golden/make_golden_configs.py config5 (CPU oracle)",
        "model": "heisenberg", "D": 3, "d": 2, "chi": chi, "seed": seed, "gs_rg_tol": 1e-10,
        "es_max_iter": 20, "es_rg_tol": 1e-8, "ad_max_iter": 4, "cases": out,
    })


def _evaluate_es(effH, effN, nrmB_cut=1e-3):
    """evaluate_es (expectation.jl:152-183) restated with numpy/scipy: the
    sorted real parts of the generalised eigenvalues of (H, N) on the
    eigenvectors of N above nrmB_cut (relative)."""
    import scipy.linalg as sl
    H = (effH + effH.conj().T) / 2
    N = (effN + effN.conj().T) / 2
    ev, P = np.linalg.eigh(N)
    idx = np.argsort(ev)[::-1]
    ev, P = ev[idx], P[:, idx]
    P = P[:, ev / ev.max() > nrmB_cut]
    H2 = P.conj().T @ H @ P
    N2 = P.conj().T @ N @ P
    es = sl.eig((H2 + H2.conj().T) / 2, (N2 + N2.conj().T) / 2, right=False)
    return np.sort(es.real)


def es_d2(seed=4, chi=8, px=1.0, py=0.0):
    """Excited-state band energies at one momentum, D=2 chi=8 Heisenberg:
    prepare_basis (optim_es.jl:34-73: ground state converged at 2 max_iter and
    rg_tol^2, normalised, E0/2 subtracted, default tangent basis), every basis
    vector's get_es_grad (optim_es.jl:127-153), effH/effN, evaluate_es."""
    A = O.random_A(2, 2, seed=seed)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=20, rg_tol=1e-6, ad_max_iter=4)
    gcfg = dict(cfg)
    gcfg.update(max_iter=2 * cfg["max_iter"], rg_tol=cfg["rg_tol"] ** 2)
    ts = O.make_ctm_tensors(A, gcfg)
    with torch.no_grad():
        ts, _ = O.run_ctm(ts, conv_fun=lambda t: O.get_gs_energy(t, H)[0])
        ts = O._detach_ts(ts).replace(Params=dict(cfg))
        ts = O.normalize_gs(ts)
        H2 = O.substract_gs_energy(ts, H)
        basis = O.get_tangent_basis(ts)
    nb = basis.shape[1]
    effH = np.zeros((nb, nb), dtype=np.complex128)
    effN = np.zeros((nb, nb), dtype=np.complex128)
    p = dict(ts.Params)
    p.update(px=px * math.pi, py=py * math.pi)
    t1 = ts.replace(Params=p)
    Bm = basis.resolve_conj().numpy()
    t0 = time.time()
    for i in range(nb):
        gH, gN = O.get_es_grad(t1, H2, basis[:, i])
        effH[:, i] = Bm.conj().T @ gH.resolve_conj().numpy() / 2
        effN[:, i] = Bm.conj().T @ gN.resolve_conj().numpy()
    print("es_d2", nb, "vectors", time.time() - t0)
    es = _evaluate_es(effH, effN)
    dump("es_d2", {
        "generator": "tests/golden/make_golden_configs.py es_d2 (CPU oracle)", "model": "heisenberg",
        "D": 2, "d": 2, "chi": chi, "seed": seed, "cfg": {k: cfg[k] for k in ("min_iter", "max_iter", "rg_tol",
                                                                            "ad_max_iter")},
        "px": px, "py": py, "nrmB_cut": 1e-3, "E0": float(complex(O.get_gs_energy(ts, H)[0]).real),
        "es": es.tolist(),
    })


def d5(iters=30, seed=1000):
    """Heisenberg D=5 chi=100 (enlarged corners 2500 x 2500), seed 1000, 30
    iterations from init_ctm1: the energy after every iteration."""
    A = O.random_A(5, 2, seed=seed)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=100, min_iter=iters, max_iter=iters, rg_tol=0.0)
    ts = O.make_ctm_tensors(A, cfg)
    traj = []
    t0 = time.time()
    with torch.no_grad():
        for i in range(iters):
            ts, s = O.rg_step(ts, 100)
            traj.append(float(complex(O.get_gs_energy(ts, H)[0]).real))
            print("d5", i, traj[-1], time.time() - t0, flush=True)
    dump("d5_chi100_30", {
        "generator": "tests/golden/make_golden_configs.py d5 (CPU oracle)", "model": "heisenberg",
        "D": 5, "d": 2, "chi": 100, "seed": seed, "energies": traj, "s_last": [float(x) for x in s.numpy()],
    })


if __name__ == "__main__":
    for name in sys.argv[1:]:
        {"config1": config1, "config2": config2, "config5": config5, "d5": d5, "es_d2": es_d2}[name]()
