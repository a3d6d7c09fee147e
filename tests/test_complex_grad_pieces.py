"""Closed forms the complex-A pullback needs, pinned against torch autograd on
the CPU (the convention is Zygote's for a real loss of a complex argument:
the gradient G satisfies dL = Re sum(conj(G) dx), i.e. G = dL/dRe x + i dL/dIm x):

* renormalisation y = x / max|x| (wrapper.jl:57) with the maximum at entry k,
  m = |x_k|:  G = g / m - e_k x_k Re(sum(conj(g) x)) / m^3;
* the bond energy E = tr(H rho) / tr(rho) (evaluation.jl:15-29), loss Re E:
  G_rho = conj(H^T - E I) / conj(tr rho);
* a loss of A and Ad = conj(A) (ctm_tensor.jl:63-69): G = G_A + conj(G_Ad).
The real pullback (csrc/ad.cu) uses the real special cases of the first two
and G_A + G_Ad for the third."""
import numpy as np
import torch


def _crandn(*shape, seed=0):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(shape, dtype=torch.float64, generator=g),
                         torch.randn(shape, dtype=torch.float64, generator=g))


def test_renormalize_backward():
    x = _crandn(5, 7, seed=1).requires_grad_(True)
    c = _crandn(5, 7, seed=2)
    m = x.abs().max()
    y = x / m
    (G,) = torch.autograd.grad((torch.conj(c) * y).sum().real, x)
    xd, g = x.detach(), c  # the cotangent of y is c
    k = int(torch.argmax(xd.abs()))
    md = xd.abs().flatten()[k]
    Gf = g / md
    Gf = Gf.flatten().clone()
    Gf[k] -= xd.flatten()[k] * (torch.conj(g) * xd).sum().real / md ** 3
    assert torch.allclose(G.flatten(), Gf, rtol=1e-12, atol=1e-14)


def test_bond_energy_seed():
    d2 = 4
    H = _crandn(d2, d2, seed=3)
    rho = _crandn(d2, d2, seed=4).requires_grad_(True)
    E = torch.trace(H @ rho) / torch.trace(rho)
    (G,) = torch.autograd.grad(E.real, rho)
    Ed = E.detach()
    Gf = torch.conj(H.T - Ed * torch.eye(d2, dtype=H.dtype)) / torch.conj(torch.trace(rho.detach()))
    assert torch.allclose(G, Gf, rtol=1e-12, atol=1e-14)


def test_A_and_conj_A_combine():
    A = _crandn(3, 4, seed=5).requires_grad_(True)
    W = _crandn(4, 3, seed=6)
    L = lambda a, ad: (torch.trace((a @ W) @ (ad @ W)) + (a * a).sum()).real
    (G,) = torch.autograd.grad(L(A, torch.conj(A)), A)
    a = A.detach().clone().requires_grad_(True)
    ad = torch.conj(A.detach()).clone().requires_grad_(True)
    ga, gad = torch.autograd.grad(L(a, ad), (a, ad))
    assert torch.allclose(G, ga + torch.conj(gad), rtol=1e-12, atol=1e-14)
    # real A: the same rule with conj the identity
    Ar = torch.randn(3, 4, dtype=torch.float64, requires_grad=True)
    Wr = W.real
    Lr = lambda a, ad: torch.trace((a @ Wr) @ (ad @ Wr)) + (a * a).sum()
    (Gr,) = torch.autograd.grad(Lr(Ar, Ar), Ar)
    a = Ar.detach().clone().requires_grad_(True)
    ad = Ar.detach().clone().requires_grad_(True)
    ga, gad = torch.autograd.grad(Lr(a, ad), (a, ad))
    assert np.allclose(Gr.numpy(), (ga + gad).numpy(), rtol=1e-12)
