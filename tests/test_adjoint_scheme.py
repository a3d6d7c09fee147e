"""The engine's projector adjoint (csrc/ad.cu `projector_backward`) restated in
numpy and checked against the oracle's full-SVD adjoint (`svd_back`,
autodiff.jl:41-74, with the eta = 1e-12 broadening), for real and complex M.

The engine never forms the full SVD.  With cotangents on the n kept triplets
only, svd_back splits into
  dM = U_t A_tt V_t^H + U_t Acol^H + Bcol V_t^H,
  Acol = M^H X_u + X_v S,  Bcol = X_u S + M X_v,
  X_u[:, j] = R_j dU[:, j],  R_j = sum over discarded a of f(s_j^2 - s_a^2) u_a u_a^H
(X_v likewise with the v's), f(x) = x / (x^2 + eta); A_tt is the kept block of
svd_back (for complex M with the extra i Im(diag(U^H dU)) S^-1 term).  R_j is
summed exactly over the discarded triplets the sketch resolved and, on their
complement, expanded in Chebyshev polynomials of B = P M M^H P over [0, b]
with the closed-form coefficients of Re 1 / (s_j^2 - i sqrt(eta) - t).  This
file checks that split, the closed-form coefficients and the stopping rule
on synthetic matrices (square and rectangular, spectrum decaying over eight
decades) to 1e-10 relative, real and complex; the CUDA path is checked
against the oracle in the GPU tests (test_energy_grad_*).

For rectangular M the reference's thin SVD weights the null space of M^H
(N1 > N2; of M when N2 > N1) by 1 / (s_j^2 + eta) per unit cotangent, while
the expansion gives it f(s_j^2) = s_j^2 / (s_j^4 + eta) like any zero
eigenvalue of B; the CUDA adjoint does the latter, a relative difference of
O(eta / s_n^4) that this file measures."""
import numpy as np
import pytest
import torch

import ipeps_oracle as O

ETA = 1e-12


def _f(x):
    return x / (x * x + ETA)


def _cheb_coefs(s2, b, m_max):
    """c[m, j]: Chebyshev coefficients over t in [0, b] of Re 1/(s2_j - i sqrt(eta) - t)."""
    z = s2 - 1j * np.sqrt(ETA)
    zeta = 2.0 * z / b - 1.0
    q = np.sqrt(zeta * zeta - 1.0 + 0j)
    # w = zeta - q with |w| < 1, formed as 1 / (zeta + q) from the larger root:
    # for s^2 >> b, zeta - q cancels to rounding noise
    q = np.where(np.abs(zeta + q) >= np.abs(zeta - q), q, -q)
    w = 1.0 / (zeta + q)
    m = np.arange(m_max)[:, None]
    c = (2.0 / b) * np.where(m == 0, 1.0, 2.0) * w[None, :] ** m / q[None, :]
    return c.real


def _resolvent_complement(Mop, Y, s2, b, tol=1e-13, m_max=400):
    """X[:, j] = f(s2_j - B) Y[:, j] on the complement (Y already projected), B = Mop."""
    c = _cheb_coefs(s2, b, m_max)
    X = c[0][None, :] * Y
    Tm1, T = Y, (2.0 / b) * Mop(Y) - Y
    for m in range(1, m_max):
        X = X + c[m][None, :] * T
        if np.abs(c[m:m + 4]).max() <= tol * np.abs(c[:m + 1]).sum(0).max():
            return X, m + 1
        Tm1, T = T, 2.0 * ((2.0 / b) * Mop(T) - T) - Tm1
    raise AssertionError("Chebyshev expansion did not reach its tolerance")


def _scheme(M, U, S, V, dU, dV, dS, n, r, null_term=False):
    """dM from n kept and r - n resolved discarded triplets (the rest by
    Chebyshev).  null_term: for rectangular M, give the null space of M^H
    (N1 > N2) or of M (N2 > N1) the reference's weight 1 / (s_j^2 + eta)
    (svd_back's (dU - U U^H dU) S^-1 V^H term of the thin SVD) instead of the
    f(s_j^2) the expansion gives every zero eigenvalue of B."""
    H = lambda X: X.conj().T
    Ut, Vt, st = U[:, :n], V[:, :n], S[:n]
    du, dv = dU[:, :n], dV[:, :n]
    s2 = st ** 2
    F = s2[None, :] - s2[:, None]
    F = F / (F * F + ETA)
    UdU = H(Ut) @ du
    J = F * UdU
    K = F * (H(Vt) @ dv)
    Att = (J + H(J)) @ np.diag(st) + np.diag(st) @ (K + H(K)) + np.diag(dS[:n])
    if np.iscomplexobj(M):
        Att = Att + np.diag(1j * np.diagonal(UdU).imag * st / (s2 + ETA))
    # resolved discarded triplets: exact
    Ur, Vr, sr = U[:, n:r], V[:, n:r], S[n:r]
    fa = _f(s2[None, :] - sr[:, None] ** 2)  # (r - n) x n
    Xu = Ur @ (fa * (H(Ur) @ du))
    Xv = Vr @ (fa * (H(Vr) @ dv))
    # complement of all resolved (kept and discarded) vectors: Chebyshev
    Ua, Va = U[:, :r], V[:, :r]
    Pu = lambda X: X - Ua @ (H(Ua) @ X)
    Pv = lambda X: X - Va @ (H(Va) @ X)
    MP = Pu(H(Pv(H(M))))  # (1 - U U^H) M (1 - V V^H)
    s_next = S[r] if r < len(S) else 0.0
    b = max(1.25 * s_next ** 2, 1e-14 * S[0] ** 2)
    assert b < s2[-1]
    Cu, tu = _resolvent_complement(lambda X: MP @ (H(MP) @ X), Pu(du), s2, b)
    Cv, tv = _resolvent_complement(lambda X: H(MP) @ (MP @ X), Pv(dv), s2, b)
    XU, XV = Xu + Cu, Xv + Cv
    if null_term and M.shape[0] != M.shape[1]:
        w = 1.0 / (s2 + ETA) - _f(s2)
        if M.shape[0] > M.shape[1]:
            XU = XU + (du - U @ (H(U) @ du)) * w[None, :]
        else:
            XV = XV + (dv - V @ (H(V) @ dv)) * w[None, :]
    Acol = H(M) @ XU + XV * st[None, :]
    Bcol = XU * st[None, :] + M @ XV
    return Ut @ Att @ H(Vt) + Ut @ H(Acol) + Bcol @ H(Vt), max(tu, tv)


def _case(N1, N2, dtype, seed):
    rng = np.random.default_rng(seed)
    k = min(N1, N2)

    def rand(*shape):
        x = rng.standard_normal(shape)
        return x + 1j * rng.standard_normal(shape) if dtype == complex else x

    Q1, _ = np.linalg.qr(rand(N1, k))
    Q2, _ = np.linalg.qr(rand(N2, k))
    s = np.logspace(0, -8, k)
    return (Q1 * s) @ Q2.conj().T


@pytest.mark.parametrize("dtype", [float, complex])
@pytest.mark.parametrize("N1,N2", [(60, 60), (70, 52)])
def test_split_adjoint_matches_svd_back(dtype, N1, N2):
    M = _case(N1, N2, dtype, seed=N1 + N2 + (dtype == complex))
    tM = torch.tensor(M)
    U, S, Vh = torch.linalg.svd(tM, full_matrices=False)
    V = Vh.mH.resolve_conj().contiguous()
    n, r = 12, 30
    rng = np.random.default_rng(7)

    def rand(*shape):
        x = rng.standard_normal(shape)
        return x + 1j * rng.standard_normal(shape) if dtype == complex else x

    k = S.shape[0]
    dU = np.zeros((N1, k), dtype=M.dtype)
    dV = np.zeros((N2, k), dtype=M.dtype)
    dS = np.zeros(k)
    dU[:, :n] = rand(N1, n)
    dV[:, :n] = rand(N2, n)
    dS[:n] = rng.standard_normal(n)
    ref = O.svd_back(U, S, V, torch.tensor(dU), torch.tensor(dS), torch.tensor(dV)).numpy()
    Un, Sn, Vn = U.numpy(), S.numpy(), V.numpy()
    dM, terms = _scheme(M, Un, Sn, Vn, dU, dV, dS, n, r, null_term=True)
    assert np.linalg.norm(dM - ref) <= 1e-10 * np.linalg.norm(ref), np.linalg.norm(dM - ref) / np.linalg.norm(ref)
    assert terms < 160  # the engine's term cap
    if N1 != N2:
        # without the null-space weight (as the CUDA adjoint runs): off by
        # O(eta / s_n^4) relative, here ~1e-6 (s_n = 0.032)
        dM0, _ = _scheme(M, Un, Sn, Vn, dU, dV, dS, n, r, null_term=False)
        dev = np.linalg.norm(dM0 - ref) / np.linalg.norm(ref)
        assert 1e-3 * ETA / Sn[n - 1] ** 4 <= dev <= 10 * ETA / Sn[n - 1] ** 4, dev


def test_chebyshev_coefficients_reproduce_the_resolvent():
    """The closed-form coefficients sum to f(s^2 - t) on [0, b] (scalar check)."""
    b = 0.3
    s2 = np.array([0.4, 0.9, 3.0])
    t = np.linspace(0, b, 101)
    tau = 2 * t / b - 1
    c = _cheb_coefs(s2, b, 200)
    T = np.cos(np.arange(200)[:, None] * np.arccos(np.clip(tau, -1, 1))[None, :])
    approx = c.T @ T
    exact = _f(s2[:, None] - t[None, :])
    assert np.abs(approx - exact).max() <= 1e-12 * np.abs(exact).max()
