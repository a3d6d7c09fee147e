"""GPU parity of the CTMRG engine (through the C ABI) against the CPU oracle.

Bars (FP64 form):
  * contraction operator and init_ctm1: 1e-12 relative (same FP64 sums, different order)
  * projector singular values: 1e-10 relative for the leading ones;
    gauge-invariant P1*P2 to 1e-8 relative
  * converged energy per site: |dE| <= 1e-10 absolute
"""
import json
import os

import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def npa(t):
    return t.detach().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


@pytest.mark.parametrize("cplx", [False, True])
def test_tcon_random_labels(engine, pkg, cplx):
    rng = np.random.default_rng(7)
    cases = [
        ([[1, 2, -1, -2], [1, 2, -3]], [(5, 4, 3, 6), (5, 4, 7)]),
        ([[-2, 1], [1, -1, -3, -4]], [(6, 5), (5, 7, 3, 2)]),
        ([[-1, -4, 1, 2, -2, -5, 3], [1, 2, -3, -6, 3]], [(4, 3, 2, 2, 3, 3, 2), (2, 2, 3, 3, 2)]),
        ([[1, 2, 3, 4, -1, -3], [1, 2, 3, 4, -2, -4]], [(3, 4, 2, 2, 2, 2), (3, 4, 2, 2, 2, 2)]),
        ([[1, 2, 3, 4, 5], [1, 2, 3, 4, 5]], [(2, 3, 2, 3, 2), (2, 3, 2, 3, 2)]),
        ([[-1, 1, -2, -3], [1, -4, -5, -6]], [(7, 5, 2, 2), (5, 6, 2, 2)]),
    ]
    for labels, shapes in cases:
        def mk(s):
            x = rng.standard_normal(s)
            if cplx:
                x = x + 1j * rng.standard_normal(s)
            return x
        A, B = mk(shapes[0]), mk(shapes[1])
        ref = npa(O.tcon([torch.tensor(A), torch.tensor(B)], labels))
        got = pkg.tcon([A, B], labels, engine=engine)
        assert got.shape == ref.shape
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_gemm_large_tcon(engine, pkg):
    """Large matrix-shaped contractions exercise both GEMM tilings and split-K."""
    rng = np.random.default_rng(3)
    for (m, k, n) in [(300, 700, 260), (40, 5000, 30), (1000, 64, 900)]:
        A = rng.standard_normal((m, k))
        B = rng.standard_normal((k, n))
        got = pkg.tcon([A, B], [[-1, 1], [1, -2]], engine=engine)
        assert np.allclose(got, A @ B, rtol=1e-12, atol=1e-11 * np.sqrt(k))
        got = pkg.tcon([A, B.T.copy()], [[-1, 1], [-2, 1]], engine=engine)
        assert np.allclose(got, A @ B, rtol=1e-12, atol=1e-11 * np.sqrt(k))


def test_projector_matches_oracle(engine, pkg):
    rng = np.random.default_rng(11)
    N, chi = 120, 30
    # decaying spectrum like an enlarged corner
    U, _ = np.linalg.qr(rng.standard_normal((N, N)))
    V, _ = np.linalg.qr(rng.standard_normal((N, N)))
    s = np.exp(-0.35 * np.arange(N))
    R1 = U @ np.diag(np.sqrt(s)) @ rng.standard_normal((N, N)) * 0.1
    R2 = np.linalg.solve(rng.standard_normal((N, N)) * 0.1, np.diag(np.sqrt(s)) @ V.T)
    P1o, P2o, So = O.get_projector(torch.tensor(R1), torch.tensor(R2), chi)
    P1, P2, S = pkg.get_projector(R1, R2, chi, engine=engine)
    So = npa(So)
    assert len(S) == len(So)
    lead = min(10, len(S))
    assert np.allclose(S[:lead], So[:lead], rtol=1e-10)
    Po = npa(P1o) @ npa(P2o)
    Pg = P1 @ P2
    assert np.linalg.norm(Pg - Po) <= 1e-8 * np.linalg.norm(Po)


def _oracle_ts_after_init(A, cfg):
    return O.make_ctm_tensors(torch.tensor(A), cfg)


def test_init_ctm1_matches(engine, pkg):
    A = npa(O.random_A(3, 2, seed=5))
    cfg = O.default_config()
    ts_o = _oracle_ts_after_init(A, cfg)
    ts = pkg.CTMTensors(A, cfg, engine=engine)
    for k in range(4):
        C, E = ts.get_CT(k + 1)
        assert np.allclose(C, npa(ts_o.Cs[k]), rtol=1e-13, atol=1e-14)
        assert np.allclose(E, npa(ts_o.Es[k]), rtol=1e-13, atol=1e-14)


def test_single_move_spectra(engine, pkg):
    A = npa(O.random_A(2, 2, seed=2))
    cfg = O.default_config()
    cfg.update(chi=12)
    ts_o = _oracle_ts_after_init(A, cfg)
    ts = pkg.CTMTensors(A, cfg, engine=engine)
    for it in range(3):
        for d, (fo, fg) in enumerate([(O.left_rg, pkg.left_rg), (O.right_rg, pkg.right_rg),
                                       (O.top_rg, pkg.top_rg), (O.bottom_rg, pkg.bottom_rg)]):
            ts_o, so = fo(ts_o, 12)
            ts, sg = fg(ts, 12)
            so = npa(so)
            assert len(sg) == len(so), (it, d)
            lead = min(8, len(so))
            assert np.allclose(sg[:lead], so[:lead], rtol=1e-10), (it, d, sg[:lead], so[:lead])


@pytest.mark.parametrize("idx", [0, 1, 2, 3])
def test_converged_energy_matches_golden(engine, pkg, idx):
    with open(os.path.join(GOLD, "ctm_energies.json")) as f:
        case = json.load(f)["cases"][idx]
    A = npa(O.random_A(case["D"], case["d"], seed=case["seed"]))
    H = O.ising(case["h"]) if case["model"] == "ising" else O.heisenberg(case["Jz"])
    H = [npa(h) for h in H]
    cfg = O.default_config()
    cfg.update(chi=case["chi"], min_iter=case["min_iter"], max_iter=case["max_iter"], rg_tol=case["rg_tol"])
    (E, Na), ts, info = pkg.compute_gs_energy(A, H, cfg, engine=engine)
    assert abs(E.real - case["E"]) <= 1e-10, (E, case["E"])
    assert info["log"][-1]["chi"] == case["chi_final"]


def test_nested_energy_and_norm(engine, pkg):
    """A few nested (excited-state) iterations: get_es_energy and get_all_norm."""
    D, chi = 2, 8
    A = O.random_A(D, 2, seed=4)
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=1, max_iter=3, rg_tol=0.0)
    ts_o = O.make_ctm_tensors(A, cfg)
    ts_o, _ = O.run_ctm(ts_o)
    g = np.random.default_rng(9)
    B = g.standard_normal(A.shape) + 1j * g.standard_normal(A.shape)
    px, py = 0.5 * np.pi, 0.25 * np.pi
    ts_o.Params.update(px=px, py=py, max_iter=2)
    ts_o = ts_o.replace(B=torch.tensor(B), Bd=torch.tensor(B).conj())
    ts_o, _ = O.run_ctm(ts_o)
    Eo = O.get_es_energy(ts_o, H).item()
    Nbo, envBo = O.get_all_norm(ts_o)

    ts = pkg.CTMTensors(npa(A), cfg, engine=engine)
    pkg.run_ctm(ts)
    ts.Params["max_iter"] = 2
    ts.set_B(B, px, py)
    pkg.run_ctm(ts)
    E = pkg.get_es_energy(ts, [npa(h) for h in H])
    Nb, envB = pkg.get_all_norm(ts)
    assert abs(E - Eo) <= 1e-9 * max(1.0, abs(Eo))
    assert abs(Nb - complex(Nbo.item())) <= 1e-9 * max(1.0, abs(complex(Nbo.item())))
    assert np.allclose(envB, npa(envBo), rtol=1e-8, atol=1e-10 * np.abs(npa(envBo)).max())


@pytest.mark.parametrize("parallel", [True, False])
def test_bench_workload_trajectory(engine, pkg, parallel):
    """The D=4 chi=64 workload (Heisenberg, 30 iterations): every
    per-iteration energy against the oracle's, with the moves in concurrent
    pairs and the energies overlapped (default) and with the four moves and
    the energies in order.  This workload does not converge: it settles into a
    period-2 cycle, which amplifies rounding-level differences of the
    truncated SVD (the order of the Jacobi rotations, the random sketch)
    instead of damping them, so its bar is 2e-10 (converging runs keep 1e-10)."""
    with open(os.path.join(GOLD, "bench_workload.json")) as f:
        g = json.load(f)
    rng = np.random.default_rng(g["seed"])
    D, d, chi = g["D"], g["d"], g["chi"]
    A = rng.standard_normal(D ** 4 * d).reshape((D, D, D, D, d), order="F")
    A = np.asfortranarray(A / np.abs(A).max())
    H = [npa(h) for h in O.heisenberg(1.0)]
    cfg = pkg.default_config()
    cfg.update(chi=chi, min_iter=30, max_iter=30, rg_tol=0.0, parallel_moves=parallel)
    ts = pkg.CTMTensors(A, cfg, engine=engine)
    ts, info = pkg.run_ctm(ts, conv_fun="energy", H=H)
    got = [l["obj"].real for l in info["log"]]
    err = max(abs(a - b) for a, b in zip(got, g["energies"]))
    assert err <= 2e-10, err


def test_d5_chi100_trajectory(engine, pkg):
    """Heisenberg D=5 chi=100 (enlarged corners 2500 x 2500, 160-column
    sketch): 8 iterations from init_ctm1 against the oracle's energies."""
    with open(os.path.join(GOLD, "d5_chi100.json")) as f:
        gold = json.load(f)
    A = npa(O.random_A(gold["D"], gold["d"], seed=gold["seed"]))
    cfg = O.default_config()
    n = len(gold["energies"])
    cfg.update(chi=gold["chi"], min_iter=n, max_iter=n, rg_tol=0.0)
    H = [npa(h) for h in O.heisenberg(1.0)]
    ts = pkg.CTMTensors(A, cfg, engine=engine)
    ts, info = pkg.run_ctm(ts, conv_fun="energy", H=H)
    traj = [l["obj"].real for l in info["log"]]
    err = max(abs(a - b) for a, b in zip(traj, gold["energies"]))
    assert err <= 1e-10, err
    ts.close()


@pytest.mark.parametrize("idx", [0, 3])
def test_early_exit_matches_sequential_loop(engine, pkg, idx):
    """run_ctm with the convergence test overlapped (the energy of iteration i
    evaluated while iteration i+1 runs, the speculative iteration rolled back on
    convergence) stops at the same iteration with the same log and environment
    shapes as the loop that evaluates every energy in order."""
    with open(os.path.join(GOLD, "ctm_energies.json")) as f:
        case = json.load(f)["cases"][idx]
    A = npa(O.random_A(case["D"], case["d"], seed=case["seed"]))
    H = O.ising(case["h"]) if case["model"] == "ising" else O.heisenberg(case["Jz"])
    H = [npa(h) for h in H]
    runs = []
    for parallel in (True, False):
        cfg = O.default_config()
        cfg.update(chi=case["chi"], min_iter=case["min_iter"], max_iter=case["max_iter"], rg_tol=case["rg_tol"],
                   parallel_moves=parallel)
        ts = pkg.CTMTensors(A, cfg, engine=engine)
        ts, info = pkg.run_ctm(ts, conv_fun="energy", H=H)
        E = pkg.get_gs_energy(ts, H)[0].real
        runs.append((info, E, [c.shape for c in ts.Cs]))
        ts.close()
    (i1, E1, s1), (i2, E2, s2) = runs
    assert i1["converged"] and i2["converged"]
    assert i1["iters"] == i2["iters"] == len(i1["log"]), (i1["iters"], i2["iters"], len(i1["log"]))
    assert s1 == s2
    assert abs(E1 - E2) <= 1e-10 and abs(E1 - case["E"]) <= 1e-10, (E1, E2, case["E"])
    assert abs(i1["log"][-1]["obj"].real - E1) <= 1e-12


def test_degenerate_rule_keeps_zero_singular_value(engine, pkg):
    """A near-product state (a product state plus 0.3 times a Gaussian tensor)
    whose enlarged corners are numerically rank 16: the cutoff keeps 16 values
    and the degenerate-pair rule (|s[17] - s[16]| < 1e-10)
    keeps a 17th (wrapper.jl:37-55), which the sketch resolves as exactly 0.  Its projector
    column must be zero, not infinite: the run stays finite and converges to
    the oracle's energy."""
    rng = np.random.default_rng(3)
    prod = np.zeros((2, 2, 2, 2, 2))
    prod[0, 0, 0, 0, :] = rng.standard_normal(2)
    A = prod + 0.3 * rng.standard_normal(prod.shape)
    A = np.asfortranarray(A / np.abs(A).max())
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=16, min_iter=4, max_iter=60, rg_tol=1e-10)
    ts_o = O.make_ctm_tensors(torch.tensor(A), cfg)
    ts_o, _ = O.run_ctm(ts_o, conv_fun=lambda x: O.get_gs_energy(x, H)[0])
    Eo = complex(O.get_gs_energy(ts_o, H)[0]).real
    (E, _), ts, info = pkg.compute_gs_energy(A, [npa(h) for h in H], cfg, engine=engine)
    assert info["converged"] and np.isfinite(E.real)
    assert abs(E.real - Eo) <= 1e-10, (E.real, Eo, [c.shape for c in ts.Cs], [tuple(c.shape) for c in ts_o.Cs])
    ts.close()


def test_projector_wide_sketch_matches_oracle(engine, pkg):
    """A sketch of 128+ columns (chi = 80 of N = 400), whose Rayleigh-Ritz SVD
    runs on the 8-CTA cluster Jacobi: leading singular values 1e-10 relative,
    P1 P2 1e-8 relative."""
    rng = np.random.default_rng(21)
    N, chi = 400, 80
    U, _ = np.linalg.qr(rng.standard_normal((N, N)))
    V, _ = np.linalg.qr(rng.standard_normal((N, N)))
    s = np.exp(-0.08 * np.arange(N))
    R1 = U @ np.diag(np.sqrt(s)) @ rng.standard_normal((N, N)) * 0.1
    R2 = np.linalg.solve(rng.standard_normal((N, N)) * 0.1, np.diag(np.sqrt(s)) @ V.T)
    P1o, P2o, So = O.get_projector(torch.tensor(R1), torch.tensor(R2), chi)
    P1, P2, S = pkg.get_projector(R1, R2, chi, engine=engine)
    So = npa(So)
    assert len(S) == len(So)
    assert np.allclose(S[:20], So[:20], rtol=1e-10)
    assert np.allclose(S, So, rtol=1e-7)
    Po = npa(P1o) @ npa(P2o)
    assert np.linalg.norm(P1 @ P2 - Po) <= 1e-8 * np.linalg.norm(Po)
