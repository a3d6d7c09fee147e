"""The 3xTF32 tcgen05 GEMM (TMA-fed, warp-specialised, split-K with FP64
partial sums) against numpy FP64.

Bar: every element within 1e-5 of sum_k |a_ik| |b_kj| (the 3xTF32 product
error is ~2^-22 per term plus FP32 accumulation inside a K split), and the
Frobenius error below 1e-5 relative for K <= 5000 - two orders of
magnitude below a single-TF32 product, which would fail both."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [
    # (opA, opB, m, n, k): tile widths 32..256, split-K, ragged edges, transposes
    ("N", "N", 1, 1, 1),
    ("N", "N", 7, 5, 33),
    ("T", "N", 130, 40, 100),
    ("N", "T", 300, 257, 70),
    ("T", "T", 129, 160, 500),
    ("N", "N", 2500, 160, 2500),   # range-finder product of the D=5 chi=100 projector
    ("T", "N", 160, 160, 2500),    # Gram-shaped
    ("N", "N", 2500, 2500, 100),   # enlarged-corner contraction
    ("N", "N", 20000, 50, 25),     # tall, small K
    ("N", "T", 1000, 1000, 4096),
]


@pytest.mark.parametrize("opA,opB,m,n,k", SHAPES)
def test_tf32x3_gemm_matches_fp64(engine, pkg, opA, opB, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((m, k) if opA == "N" else (k, m))
    B = rng.standard_normal((k, n) if opB == "N" else (n, k))
    C0 = rng.standard_normal((m, n))
    Am = A if opA == "N" else A.T
    Bm = B if opB == "N" else B.T
    for alpha, beta in [(1.0, 0.0), (-0.5, 2.0)]:
        C = pkg.host.gemm_tf32x3(opA, opB, A, B, alpha=alpha, beta=beta, C=C0, engine=engine)
        ref = alpha * (Am @ Bm) + beta * C0
        bound = abs(alpha) * (np.abs(Am) @ np.abs(Bm))
        err = np.abs(C - ref)
        assert np.all(err <= 1e-5 * bound + 1e-12 * abs(beta) * np.abs(C0)), (err / (bound + 1e-300)).max()
        assert np.linalg.norm(C - ref) <= 1e-5 * np.linalg.norm(alpha * (Am @ Bm)), (
            np.linalg.norm(C - ref) / np.linalg.norm(alpha * (Am @ Bm)))


def test_tf32x3_repeatable(engine, pkg):
    """The same product twice gives identical bits (deterministic split-K sum)."""
    rng = np.random.default_rng(5)
    A = rng.standard_normal((700, 3000))
    B = rng.standard_normal((3000, 90))
    C1 = pkg.host.gemm_tf32x3("N", "N", A, B, engine=engine)
    C2 = pkg.host.gemm_tf32x3("N", "N", A, B, engine=engine)
    assert np.array_equal(C1, C2)
