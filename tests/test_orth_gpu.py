"""The projector's orthonormalisation (shifted CholeskyQR, csrc/projector.cu
`orth`) through ``ipeps_orth``: the range-finder step that stands in for the
Q factor of the reference's full SVD (ctmrg.jl:257).  It exercises the
register-resident Cholesky (k <= 160), the blocked Cholesky (larger k) and the
row-parallel triangular solve directly, against numpy's QR:

* Q^T Q = I to 1e-14 and Q R = Y to 1e-14 relative (sCholQR3 on a
  well-conditioned Y); one pass (shifted) orthogonal to 1e-6, two to 1e-14;
* R equals numpy's R up to the signs of its rows, to 1e-12 relative (R has a
  positive diagonal);
* ill-conditioned Y (singular values 1 .. 1e-12; the first pass is shifted):
  Q^T Q = I to 1e-13 after three passes; rank-deficient Y (rank k/2): Q^T Q = I
  to 1e-10 (the null directions are rounding noise); in both the range of Y
  lies inside range(Q) to 1e-13.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,k", [(300, 5), (1000, 33), (2500, 128), (2500, 160), (1200, 200)])
def test_orth_matches_numpy_qr(engine, pkg, N, k):
    rng = np.random.default_rng(N + k)
    Y = rng.standard_normal((N, k))
    Q, R = pkg.orth(Y, 3, engine=engine)
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-14 * k ** 0.5
    assert np.linalg.norm(Q @ R - Y) <= 1e-14 * np.linalg.norm(Y) * k ** 0.5
    assert np.allclose(np.tril(R, -1), 0.0)
    assert (np.diag(R) > 0).all()
    _, Rn = np.linalg.qr(Y)
    Rn = Rn * np.sign(np.diag(Rn))[:, None]
    assert np.linalg.norm(R - Rn) <= 1e-12 * np.linalg.norm(Rn)
    # one shifted pass is orthogonal only to the shift's level, ~11 (N k + k^2) u
    # trace(G) / s_min(Y)^2 (a CPU restatement: 1e-11 at k = 5 .. 1e-7 at k = 160);
    # the unshifted second pass restores the rounding level
    for passes, bar in ((1, 1e-6), (2, 1e-14 * k ** 0.5)):
        Qp, Rp = pkg.orth(Y, passes, engine=engine)
        assert np.abs(Qp.T @ Qp - np.eye(k)).max() <= bar, passes
        assert np.linalg.norm(Qp @ Rp - Y) <= 1e-13 * np.linalg.norm(Y)


@pytest.mark.parametrize("k", [64, 160])
def test_orth_ill_conditioned_and_rank_deficient(engine, pkg, k):
    rng = np.random.default_rng(7 * k)
    N = 2000
    # singular values from 1 down to 1e-12 (as a sketch after power iterations)
    U, _ = np.linalg.qr(rng.standard_normal((N, k)))
    V, _ = np.linalg.qr(rng.standard_normal((k, k)))
    Y = (U * np.logspace(0, -12, k)) @ V.T
    Q, R = pkg.orth(Y, 3, engine=engine)
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-13
    assert np.linalg.norm(Y - Q @ (Q.T @ Y)) <= 1e-13 * np.linalg.norm(Y)
    # rank k/2: the shifted first pass keeps R invertible, Q stays orthonormal
    Yr = rng.standard_normal((N, k // 2)) @ rng.standard_normal((k // 2, k))
    Q, R = pkg.orth(Yr, 3, engine=engine)
    assert np.isfinite(Q).all() and np.isfinite(R).all()
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-10  # a CPU restatement gives 1.3e-11 at k = 160
    assert np.linalg.norm(Yr - Q @ (Q.T @ Yr)) <= 1e-13 * np.linalg.norm(Yr)
