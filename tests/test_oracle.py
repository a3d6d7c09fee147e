"""CPU tests of the oracle against the reference's own pins.

Pins (reference test files, read as text):
  * test/test_model.jl:9-16, test/test_ctmrg.jl:5-12: honeycomb XX init state,
    default config: real(e0)/8 == -0.16349 (atol 1e-5)
  * test/test_model.jl:78-83: GHZ-Q state with honeycomb(1,1): same value
  * test/test_nest.jl:20-26: nested product rule
  * test/test_tcon.jl:5-15: tcon == einsum
"""
import json
import os

import numpy as np
import pytest
import torch

import ipeps_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_tcon_matches_einsum():
    g = torch.Generator().manual_seed(0)
    A = torch.rand(5, 5, 5, 5, generator=g, dtype=torch.float64)
    B = torch.rand(5, 5, 5, generator=g, dtype=torch.float64)
    r0 = torch.einsum("abmn,abk->mnk", A, B)
    r1 = O.tcon([A, B], [[1, 2, -1, -2], [1, 2, -3]])
    assert torch.allclose(r0, r1)


def test_nested_product_rule():
    g = torch.Generator().manual_seed(1)
    A = [torch.rand(5, 5, 5, generator=g, dtype=torch.float64) for _ in range(4)]
    B = [torch.rand(5, 5, 5, generator=g, dtype=torch.float64) for _ in range(4)]
    A1, B1 = O.NestedTensor(A), O.NestedTensor(B)
    ind = [[-1, 1, 2], [1, 2, -2]]
    C = O.tcon([A1, B1], ind)
    t = lambda a, b: O.tcon([a, b], ind)
    assert torch.equal(C[1], t(A[0], B[0]))
    assert torch.allclose(C[2], t(A[0], B[1]) + t(A[1], B[0]))
    assert torch.allclose(C[3], t(A[0], B[2]) + t(A[2], B[0]))
    assert torch.allclose(C[4], t(A[0], B[3]) + t(A[3], B[0]) + t(A[1], B[2]) + t(A[2], B[1]))


def test_empty_absorbs():
    A = O.NestedTensor([torch.ones(2, 2, dtype=torch.float64), None, None, None])
    B = O.NestedTensor([torch.ones(2, 2, dtype=torch.float64), torch.ones(2, 2, dtype=torch.float64), None, None])
    C = O.tcon([A, B], [[-1, 1], [1, -2]])
    assert C[3] is None and C[4] is None and C[2] is not None


def test_freshape_is_column_major():
    x = torch.arange(24, dtype=torch.float64)
    y = O.freshape(x, 2, 3, 4)
    # Julia: reshape(0:23, 2,3,4)[i,j,k] = i + 2j + 6k (0-based)
    assert y[1, 2, 3].item() == 1 + 2 * 2 + 6 * 3


def test_honeycomb_known_answer():
    A = O.init_hb_gs(2, p1=0.24, p2=0, dir="XX")
    H = O.honeycomb(1, 1, dir="XX")
    e0, _ = O.compute_gs_energy(A, H, O.default_config())
    assert abs(e0.real.item() / 8 - (-0.16349)) < 1e-5


def test_ghz_known_answer():
    A = O.get_Q_ghz()
    H = O.honeycomb(1, 1)
    e0, _ = O.compute_gs_energy(A, H, O.default_config())
    assert abs(e0.real.item() / 8 - (-0.16349)) < 1e-5


def test_golden_fixtures_match_oracle():
    """The committed fixtures (tests/golden/make_golden.py) reproduce exactly."""
    with open(os.path.join(GOLD, "ctm_energies.json")) as f:
        gold = json.load(f)
    for case in gold["cases"][:2]:
        A = O.random_A(case["D"], case["d"], seed=case["seed"])
        H = O.ising(case["h"]) if case["model"] == "ising" else O.heisenberg(case["Jz"])
        cfg = O.default_config()
        cfg.update(chi=case["chi"], min_iter=case["min_iter"], max_iter=case["max_iter"], rg_tol=case["rg_tol"])
        e0, _ = O.compute_gs_energy(A, H, cfg)
        assert abs(complex(e0).real - case["E"]) < 1e-12


def test_gradient_matches_finite_differences():
    """No gradient pin exists in the reference (test/test_svd_ad.jl is empty):
    the oracle's reference-adjoint gradient is checked by central differences.
    The eta = 1e-12 broadening of svd_back (autodiff.jl:41-48) makes the
    agreement approximate (observed ~1e-5 relative), so the bound is 1e-3."""
    torch.manual_seed(0)
    A = O.random_A(2, 2, seed=1)
    H = O.ising(2.0)
    cfg = O.default_config()
    cfg.update(chi=8, max_iter=30, min_iter=4, rg_tol=1e-10)
    E, g, ts = O.energy_and_grad(A, H, cfg)
    x0 = O.renormalize(A)

    def f(x):
        with torch.no_grad():
            return O.run_gs(ts, H, x).real.item() if torch.is_complex(O.run_gs(ts, H, x)) else O.run_gs(ts, H, x).item()

    for k in range(3):
        v = torch.randn(A.shape, dtype=torch.float64)
        h = 1e-6
        fd = (f(x0 + h * v) - f(x0 - h * v)) / (2 * h)
        an = (g * v).sum().item()
        assert abs(fd - an) <= 1e-3 * abs(an) + 1e-8


def test_complex_gradient_matches_finite_differences():
    """The reference differentiates a ComplexF64 A as well (test/optim_gs.jl:17-25:
    randn(ComplexF64, D,D,D,D,d) with the Ising Hamiltonian).  The oracle's
    gradient follows Zygote's convention for a real loss of a complex argument,
    g = dE/dRe A + i dE/dIm A, so a step h v changes E by h Re(sum(conj(g) v));
    checked by central differences along complex directions (bound as in the
    real case)."""
    torch.manual_seed(0)
    g0 = torch.Generator().manual_seed(3)
    A = torch.complex(torch.randn((2, 2, 2, 2, 2), dtype=torch.float64, generator=g0),
                      torch.randn((2, 2, 2, 2, 2), dtype=torch.float64, generator=g0))
    H = O.ising(2.0)
    cfg = O.default_config()
    cfg.update(chi=8, max_iter=30, min_iter=4, rg_tol=1e-10)
    E, g, ts = O.energy_and_grad(A, H, cfg)
    assert torch.is_complex(g) and g.shape == A.shape
    x0 = O.renormalize(A)

    def f(x):
        with torch.no_grad():
            return O.run_gs(ts, H, x).real.item()

    for k in range(3):
        v = torch.complex(torch.randn(A.shape, dtype=torch.float64), torch.randn(A.shape, dtype=torch.float64))
        h = 1e-6
        fd = (f(x0 + h * v) - f(x0 - h * v)) / (2 * h)
        an = (torch.conj(g) * v).sum().real.item()
        assert abs(fd - an) <= 1e-3 * abs(an) + 1e-8, (k, fd, an)
