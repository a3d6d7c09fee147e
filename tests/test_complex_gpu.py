"""Complex iPEPS tensors and general projector shapes on the GPU.

test/test_model.jl:9-16 and :78-83 converge CTMRG for two ComplexF64
honeycomb states (d = 4) with the default config (chi = 32) and check
real(E)/8 = -0.16349 +- 1e-5.  Here the same cases run through the C ABI
(complex range finder, complex CholeskyQR and complex one-sided Jacobi in the
projector) and are compared with (a) the reference's known answer and (b)
the CPU oracle's per-iteration energies (tests/golden/honeycomb_kat.json,
written by tests/golden/make_golden.py --honeycomb).  Their environments grow
unevenly in the first iterations, so M = R1 R2 is rectangular there, and
their spectra reach down to the 1e-12 relative cutoff.

Bars: every iterate within 1e-9 of the oracle (|dE|/8 <= 1.25e-10 per site;
both FP64), the known answer to 1e-5; projector singular values 1e-10
relative, gauge-invariant P1 P2 1e-8 relative.
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


def kat_case(name):
    if name == "init_hb_gs_XX":
        return O.init_hb_gs(2, p1=0.24, p2=0, dir="XX"), O.honeycomb(1, 1, dir="XX")
    return O.get_Q_ghz(), O.honeycomb(1, 1)


@pytest.mark.parametrize("name", ["init_hb_gs_XX", "ghz"])
def test_honeycomb_known_answer(engine, pkg, name):
    with open(os.path.join(GOLD, "honeycomb_kat.json")) as f:
        gold = {c["name"]: c for c in json.load(f)["cases"]}[name]
    A, H = kat_case(name)
    A = npa(A)
    H = [npa(h) for h in H]
    assert np.iscomplexobj(A)
    cfg = O.default_config()
    (E, Na), ts, info = pkg.compute_gs_energy(A, H, cfg, engine=engine)
    traj = [l["obj"].real for l in info["log"]]
    assert len(traj) == gold["iters"]
    err = max(abs(a - b) for a, b in zip(traj, gold["trajectory"]))
    assert err <= 1e-9, (name, err)
    assert abs(E.real - gold["E"][0]) <= 1e-9, (E, gold["E"])
    assert abs(E.real / 8 - (-0.16349)) < 1e-5, E.real / 8
    ts.close()


def _crandn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _check_projector(pkg, engine, R1, R2, chi):
    P1o, P2o, So = O.get_projector(torch.tensor(R1), torch.tensor(R2), chi)
    P1, P2, S = pkg.get_projector(R1, R2, chi, engine=engine)
    So = npa(So)
    assert P1.shape == (R1.shape[1], len(S)) and P2.shape == (len(S), R1.shape[1])
    assert len(S) == len(So), (len(S), len(So))
    lead = min(10, len(S))
    assert np.allclose(S[:lead], So[:lead], rtol=1e-10), (S[:lead], So[:lead])
    Po = npa(P1o) @ npa(P2o)
    assert np.linalg.norm(P1 @ P2 - Po) <= 1e-8 * np.linalg.norm(Po)


@pytest.mark.parametrize("N, chi, rank", [(120, 30, None), (16, 32, 4), (128, 32, 40)])
def test_complex_projector_matches_oracle(engine, pkg, N, chi, rank):
    """ipeps_projector_c vs the oracle's get_projector (LAPACK SVD of R1 R2).
    rank < N makes M = R1 R2 rank deficient, so the kept count comes from the
    1e-12 relative cutoff."""
    rng = np.random.default_rng(5 + N)
    U, _ = np.linalg.qr(_crandn(rng, N, N))
    V, _ = np.linalg.qr(_crandn(rng, N, N))
    s = np.exp(-0.35 * np.arange(N))
    if rank is not None:
        s[rank:] = 0.0
    R1 = U @ np.diag(np.sqrt(s)) @ _crandn(rng, N, N) * 0.1
    R2 = np.linalg.solve(_crandn(rng, N, N) * 0.1, np.diag(np.sqrt(s)) @ V.conj().T)
    _check_projector(pkg, engine, R1, R2, chi)


@pytest.mark.parametrize("cplx", [False, True])
def test_rectangular_projector_matches_oracle(engine, pkg, cplx):
    """M = R1 R2 rectangular (N1 x N2), as in the first iterations from
    init_ctm1 when the corner dimensions of the environment still differ."""
    rng = np.random.default_rng(17)
    N1, K1, N2, chi = 44, 76, 56, 32
    rn = (lambda *s: _crandn(rng, *s)) if cplx else (lambda *s: rng.standard_normal(s))
    U, _ = np.linalg.qr(rn(N1, N1))
    V, _ = np.linalg.qr(rn(N2, N2))
    s = np.exp(-0.5 * np.arange(N1))
    R1 = U @ np.diag(np.sqrt(s)) @ rn(N1, K1) * 0.1
    R2 = rn(K1, N1) @ np.diag(np.sqrt(s)) @ V[:, :N1].conj().T * 0.1
    _check_projector(pkg, engine, R1, R2, chi)


def test_real_projector_rank_deficient(engine, pkg):
    """Real M = R1 R2 of exact rank 4 (like the first move from init_ctm1 of a
    low-entanglement state): the kept count must equal the oracle's."""
    rng = np.random.default_rng(12)
    N, chi = 16, 32
    U, _ = np.linalg.qr(rng.standard_normal((N, N)))
    V, _ = np.linalg.qr(rng.standard_normal((N, N)))
    s = np.exp(-0.35 * np.arange(N))
    s[4:] = 0.0
    R1 = U @ np.diag(np.sqrt(s)) @ rng.standard_normal((N, N)) * 0.1
    R2 = np.linalg.solve(rng.standard_normal((N, N)) * 0.1, np.diag(np.sqrt(s)) @ V.T)
    _check_projector(pkg, engine, R1, R2, chi)
