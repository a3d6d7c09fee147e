"""The engine's FP64 GEMM (DMMA tensor-core kernel, gemm_dmma.cu) through the
C ABI against a numpy FP64 product: every op combination, edge tiles (sizes
that are not multiples of the tiles), odd leading dimensions (8-byte copies;
even ones take 16-byte copies),
split-K shapes (few output tiles, long K) and beta != 0.

Bar: |C - C_ref| <= 2 k eps (|A| |B|)_ij + 2 eps |beta C|_ij per entry, the
bound of any FP64 summation order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps

CASES = [
    # m, n, k, beta != 0
    (1, 1, 1, 0),
    (7, 5, 3, 1),
    (64, 64, 16, 0),
    (130, 70, 33, 1),
    (2500, 160, 2500, 0),   # projector range finder: few output tiles, long K (split-K)
    (160, 160, 2500, 0),    # Gram matrix shape
    (161, 157, 3001, 1),    # split-K with edge tiles and beta (23 splits)
    (97, 33, 20000, 1),     # two output tiles, 156 splits
    (1000, 1200, 100, 0),   # many output tiles (128x128 kernel)
    (1001, 1203, 101, 1),   # the same with odd sizes (odd leading dimensions)
    (40000, 50, 25, 0),     # tall and narrow (128x64 tiles): the contractions with A
    (40001, 49, 25, 1),     # the same, odd
    (50, 40000, 25, 0),     # short and wide (64x128 tiles)
]


@pytest.mark.parametrize("opA", ["N", "T"])
@pytest.mark.parametrize("opB", ["N", "T"])
@pytest.mark.parametrize("case", CASES)
def test_gemm_f64_matches_numpy(engine, pkg, opA, opB, case):
    m, n, k, pad = case
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    ar, ac = (m, k) if opA == "N" else (k, m)
    br, bc = (k, n) if opB == "N" else (n, k)
    A = np.asfortranarray(rng.standard_normal((ar, ac)))
    B = np.asfortranarray(rng.standard_normal((br, bc)))
    C = rng.standard_normal((m, n))
    alpha, beta = 0.75, (0.0 if pad == 0 else -1.5)
    opa = (lambda x: x) if opA == "N" else (lambda x: x.T)
    opb = (lambda x: x) if opB == "N" else (lambda x: x.T)
    ref = alpha * (opa(A) @ opb(B)) + beta * C
    out = pkg.host.gemm_f64(opA, opB, A, B, alpha=alpha, beta=beta, C=C, engine=engine)
    bound = 2 * k * EPS * abs(alpha) * (np.abs(opa(A)) @ np.abs(opb(B))) + 2 * EPS * np.abs(beta * C) + 1e-300
    assert np.all(np.abs(out - ref) <= bound), float(np.max(np.abs(out - ref) / bound))


def test_gemm_f64_split_k_is_deterministic(engine, pkg):
    """The split-K partial products are summed in split order, whatever order
    the CTAs ran in: repeated products are bitwise equal."""
    rng = np.random.default_rng(5)
    A = np.asfortranarray(rng.standard_normal((2500, 160)))
    B = np.asfortranarray(rng.standard_normal((2500, 160)))
    outs = [pkg.host.gemm_f64("T", "N", A, B, engine=engine) for _ in range(4)]
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    ref = A.T @ B
    bound = 2 * 2500 * EPS * (np.abs(A.T) @ np.abs(B))
    assert np.all(np.abs(outs[0] - ref) <= bound)
